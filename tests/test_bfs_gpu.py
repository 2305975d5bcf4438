"""Parity of the sm_100a BFS engine with the CPU oracle, through the C ABI.

Depths must be bit-exact (integer work); parents must form a valid BFS tree.
"""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu

DIRS = [S.DIR_ALPHABETA, S.DIR_PUSH, S.DIR_PULL]


def check_run(csr, g, src, gt=None, direction=S.DIR_ALPHABETA, unreached=S.UNREACHED, tcsr=None, **kw):
    eng = S.Engine(g, gt, direction=direction, unreached=unreached, **kw)
    depth, parent, st = eng.bfs(src, parents=True)
    ref = O.bfs(csr.idx, csr.ngh, src, unreached)
    mism = np.flatnonzero(depth != ref)
    assert mism.size == 0, f"src {src} dir {direction}: {mism.size} mismatches, first v={mism[0]} " \
                           f"gpu={depth[mism[0]]} cpu={ref[mism[0]]}"
    rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent, unreached)
    assert rc == 0, f"invalid tree code {rc} at {bad}"
    assert st.reached == int((ref != unreached).sum())
    trace = eng.trace()
    eng.close()
    return depth, st, trace


@pytest.fixture(scope="module")
def rmat16():
    csr = S.Csr.rmat(16, 16, seed=G.SEED + 0)
    return csr, S.PagedGraph.from_csr(csr)  # 10 Mi-word pages, like the reference default


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
@pytest.mark.parametrize("direction", DIRS)
def test_rmat16_max_degree_source(rmat16, direction, use_graph):
    csr, g = rmat16
    src = int(np.argmax(csr.degree()))
    _, st, tr = check_run(csr, g, src, direction=direction, use_graph=use_graph)
    assert [t["direction"] for t in tr][0] == 0
    if direction == S.DIR_PUSH:
        assert st.pull_levels == 0
    if direction == S.DIR_PULL:
        assert st.push_levels == 1


def test_graph_and_host_loop_take_the_same_decisions():
    csr = S.Csr.rmat(15, 16, seed=G.SEED + 8)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 15)
    for src in G.sources(csr, 3, 8):
        _, _, t1 = check_run(csr, g, src, use_graph=0)
        _, _, t2 = check_run(csr, g, src, use_graph=2)
        assert [(t["direction"], t["next"], t["edges_inspected"]) for t in t1] == \
               [(t["direction"], t["next"], t["edges_inspected"]) for t in t2]


def test_async_runs_back_to_back():
    """Enqueued graph-mode runs (no host sync in between) give the oracle's depths."""
    import torch

    csr = S.Csr.rmat(14, 16, seed=G.SEED + 9)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    stream = torch.cuda.current_stream()
    eng = S.Engine(g, stream=stream.cuda_stream)
    srcs = G.sources(csr, 4, 9)
    outs = [torch.empty(csr.V, dtype=torch.int32, device="cuda") for _ in srcs]
    for s, o in zip(srcs, outs):
        eng.bfs_async(s, o.data_ptr())
    eng.sync()
    for s, o in zip(srcs, outs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), O.bfs(csr.idx, csr.ngh, s))
    tr = eng.trace()  # trace of the last run, read back on demand
    assert 1 + sum(t["next"] for t in tr) == int((O.bfs(csr.idx, csr.ngh, srcs[-1]) != S.UNREACHED).sum())
    eng.close()


def test_enqueue_pipelines_host_output():
    """Pipelined runs into page-locked host buffers (two device buffers reused
    in turn, copies on a second stream) give the oracle's depths, interleaved
    with plain synchronous runs; the host loop refuses the pipelined call."""
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 10)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    eng = S.Engine(g)
    srcs = G.sources(csr, 5, 10)
    bufs = [S.PinnedArray(csr.V) for _ in srcs]
    for b in bufs:
        b.array.fill(0xDEADBEEF)
    for s, b in zip(srcs[:3], bufs[:3]):
        eng.bfs_enqueue(s, b.array)
    mid, _, _ = eng.bfs(srcs[0])  # a synchronous run between pipelined ones
    for s, b in zip(srcs[3:], bufs[3:]):
        eng.bfs_enqueue(s, b.array)
    eng.sync()
    assert np.array_equal(mid, O.bfs(csr.idx, csr.ngh, srcs[0]))
    for s, b in zip(srcs, bufs):
        assert np.array_equal(b.array, O.bfs(csr.idx, csr.ngh, s)), f"src {s}"
    eng.close()
    hl = S.Engine(g, use_graph=2)
    with pytest.raises(S.ScaphError):
        hl.bfs_enqueue(srcs[0], bufs[0].array)
    hl.close()
    for b in bufs:
        b.close()


def test_rmat16_reference_sentinel(rmat16):
    """Reference convention: unreached = 63 (app/bfs.cu:18), bit-exact with bfs::check's rule."""
    csr, g = rmat16
    src = int(np.argmax(csr.degree()))
    check_run(csr, g, src, unreached=S.REF_UNREACHED)


def test_rmat_multipage_random_sources():
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 1)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 13)
    assert g.npages > 10
    for i, src in enumerate(G.sources(csr, 6, 1)):
        check_run(csr, g, src, direction=DIRS[i % 3])


@pytest.mark.parametrize("block", [128, 256, 512])
def test_block_sizes(block):
    csr = S.Csr.rmat(13, 8, seed=G.SEED + 2)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 12)
    for src in G.sources(csr, 2, 2):
        check_run(csr, g, src, block_size=block)


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_deep_path_and_cap(use_graph):
    """A 300-vertex path: native depths go to 299; with the reference sentinel
    63 the reference semantics cap reachability at depth 62."""
    csr = G.path(300)
    g = S.PagedGraph.from_csr(csr, pagesize_words=256)
    _, st, _ = check_run(csr, g, 0, direction=S.DIR_PUSH, use_graph=use_graph)
    assert st.levels == 300
    check_run(csr, g, 150, direction=S.DIR_PULL, use_graph=use_graph)
    d, _, _ = check_run(csr, g, 0, unreached=S.REF_UNREACHED, use_graph=use_graph)
    assert d.max() == 63 and (d == 62).sum() == 1


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_deeper_than_level_cap_is_an_error(use_graph):
    """The engine's level loop keeps one counter record per level (4096): a
    path longer than that returns SCAPH_EUNSUPPORTED instead of depths with
    the far end left unreached; the multi-source loop does the same."""
    csr = G.path(4200)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 15)
    eng = S.Engine(g, direction=S.DIR_PUSH, use_graph=use_graph)
    with pytest.raises(S.ScaphError) as ex:
        eng.bfs(0)
    assert ex.value.code == S.EUNSUPPORTED and "deeper than 4096" in str(ex.value)
    # from the middle the depths reach 2100 (2101 levels, the last finding
    # nothing): exact
    d, _, st = eng.bfs(2100)
    assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, 2100)) and st.levels == 2101
    with pytest.raises(S.ScaphError) as ex:
        eng.msbfs([0, 5])
    assert ex.value.code == S.EUNSUPPORTED
    eng.close()


def test_isolated_source_and_ragged_V():
    csr = G.random_graph(1001, 900, seed=3)  # V not a multiple of 32, isolated vertices
    g = S.PagedGraph.from_csr(csr, pagesize_words=512)
    iso = [int(v) for v in np.flatnonzero(csr.degree() == 0)[:2]]
    for src in iso + G.sources(csr, 3, 3) + [1000]:
        check_run(csr, g, src)


def test_giant_vertex_chunks():
    """A hub of degree > 4096 goes through the giant-chunk kernel."""
    csr = G.star(20000, center=77)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 16)
    check_run(csr, g, 77, direction=S.DIR_PUSH)
    check_run(csr, g, 5, direction=S.DIR_PUSH)
    check_run(csr, g, 5)


@pytest.mark.parametrize("direction", DIRS)
def test_directed_powerlaw_with_transpose(direction):
    csr = S.Csr.powerlaw(20000, 300000, 1.9, 2000, seed=G.SEED + 3)
    t = csr.transpose()
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    gt = S.PagedGraph.from_csr(t, pagesize_words=1 << 14)
    for src in G.sources(csr, 3, 4):
        check_run(csr, g, src, gt=gt, direction=direction)


def test_web_graph():
    csr = S.Csr.web(50000, 600000, 2.1, 5000, 4096, 0.9, seed=G.SEED + 5)
    t = csr.transpose()
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 15)
    gt = S.PagedGraph.from_csr(t, pagesize_words=1 << 15)
    for src in G.sources(csr, 3, 5):
        check_run(csr, g, src, gt=gt)


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_trace_and_page_histogram(use_graph):
    """Per-level trace adds up, and the fused per-page frontier histogram equals
    get_page_info's (src/gpu_engine.cuh:397-441) restated in the oracle."""
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 6)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    src = G.sources(csr, 1, 6)[0]
    if True:
        # resident runs record the histograms only on request
        plain = S.Engine(g, use_graph=use_graph)
        plain.bfs(src)
        with pytest.raises(S.ScaphError):
            plain.page_hist(1)
        plain.close()
    eng = S.Engine(g, use_graph=use_graph, record_features=1)
    depth, _, st = eng.bfs(src)
    tr = eng.trace()
    assert len(tr) == st.levels
    assert 1 + sum(t["next"] for t in tr) == st.reached
    deg = csr.degree()
    for lvl in range(1, st.levels + 1):
        stat = (depth == lvl).astype(np.uint8)
        nodes, datas, _, _ = O.page_stats(g.page_list(), stat, deg)
        hn, hd = eng.page_hist(lvl)
        assert np.array_equal(hn, nodes) and np.array_equal(hd, datas), f"level {lvl}"
        if lvl < st.levels:
            assert tr[lvl]["frontier"] == stat.sum()
    eng.close()


def test_pages_from_files(tmp_path):
    """Engine over pages read back from disk (the pagegencsr file set)."""
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 7)
    prefix = str(tmp_path / "g")
    csr.write(prefix)
    csr.write_pages(prefix, 1 << 13)
    g = S.PagedGraph.open(prefix)
    for src in G.sources(csr, 2, 7):
        check_run(csr, g, src)


def test_bad_source_is_an_error(rmat16):
    csr, g = rmat16
    eng = S.Engine(g)
    with pytest.raises(S.ScaphError) as ei:
        eng.bfs(csr.V)
    assert ei.value.code == S.EINVAL
    eng.close()


def test_grown_page_for_a_giant_vertex(tmp_path):
    """Pages written with growth (the page enlarged to hold a list longer
    than the requested page) run through the engine, resident and out of
    core, with exact depths."""
    csr = G.star(5000, center=17)
    extra = G.random_graph(5000, 8000, seed=9)
    csr = G.csr_from_edges(5000, np.concatenate([np.repeat(np.arange(5000), np.diff(csr.idx).astype(np.int64)),
                                                 np.repeat(np.arange(5000), np.diff(extra.idx).astype(np.int64))]),
                           np.concatenate([csr.ngh, extra.ngh]))
    csr.write(str(tmp_path / "g"))
    ps = S.pages_write_stream(str(tmp_path / "g"), str(tmp_path / "p"), 2048, grow=True)
    assert ps > 2048
    g = S.PagedGraph.open(str(tmp_path / "p"))
    for pool in (0, 2 * ps * 4):
        eng = S.Engine(g, pool_bytes=pool)
        for src in (17, 3, 4999):
            d, _, _ = eng.bfs(src)
            assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src))
        eng.close()
