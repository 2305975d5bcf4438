"""Parity at larger sizes: an RMAT-21 graph cut into ~600 pages (more than
the 512 page-table entries and 1024 coarse-index buckets the level kernels
stage in shared memory, so they read the tables from global memory), RMAT-22
at the reference's 10 Mi-word pages, and a directed power-law graph of 2.2M
vertices with its transposed pages, in HBM and streamed through a small
page pool.  Single-source runs, multi-source batches and the out-of-core
pager are compared bit for bit with the CPU oracle (OpenMP restatement of
bfs::check, app/bfs.cu:70-101)."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu


def _same(csr, src, depth, unreached=S.UNREACHED):
    ref = O.bfs_omp(csr.idx, csr.ngh, int(src), unreached)
    bad = np.flatnonzero(depth != ref)
    assert bad.size == 0, f"src {src}: {bad.size} mismatches, v={bad[0]} gpu={depth[bad[0]]} cpu={ref[bad[0]]}"


@pytest.fixture(scope="module")
def rmat21():
    csr = S.Csr.rmat(21, 16, seed=G.SEED + 60, scramble=True)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 16)
    assert g.npages > 512
    return csr, g


@pytest.fixture(scope="module")
def powerlaw2m():
    csr = S.Csr.powerlaw(2_200_000, 33_000_000, 1.9, 1 << 15, seed=G.SEED + 61)
    tcsr = csr.transpose()
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 18)
    gt = S.PagedGraph.from_csr(tcsr, pagesize_words=1 << 18)
    return csr, g, gt


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_rmat21_many_pages(rmat21, use_graph):
    csr, g = rmat21
    eng = S.Engine(g, use_graph=use_graph)
    srcs = G.sources(csr, 3, 60) + [int(np.argmax(csr.degree()))]
    pulls = 0
    for src in srcs:
        depth, parent, st = eng.bfs(src, parents=True)
        _same(csr, src, depth)
        rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
        assert rc == 0, f"invalid BFS tree (code {rc} at {bad})"
        pulls += st.pull_levels
    assert pulls > 0
    eng.close()


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_rmat21_sparse_push_windows(rmat21, use_graph):
    """Every level pushes through the sparse front-end (push_sparse_ratio 1)
    with one CTA per SM: a CTA's run of frontier words (443 words, up to
    14 K vertices) then holds more frontier vertices than its 4096-entry
    queue at the big levels, so the queue is filled and expanded in
    windows.  Depths bit-exact, parents a valid BFS tree, with and without
    deferred claims."""
    csr, g = rmat21
    for defer in (-1, 1):
        eng = S.Engine(g, use_graph=use_graph, direction=S.DIR_PUSH, ctas_per_sm=1, push_sparse_ratio=1,
                       push_defer_edges=defer)
        for src in G.sources(csr, 2, 68) + [int(np.argmax(csr.degree()))]:
            depth, parent, st = eng.bfs(src, parents=defer < 0)
            _same(csr, src, depth)
            assert st.pull_levels == 0
            if defer < 0:
                rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
                assert rc == 0, f"invalid BFS tree (code {rc} at {bad})"
        eng.close()


@pytest.mark.parametrize("use_graph", [0, 2], ids=["graph", "hostloop"])
def test_rmat21_pull_runs_windows(rmat21, use_graph):
    """Every level after the first pulls, each as a sparse level read in one
    run of visited words per CTA (pull_gather_ratio 1), with one CTA per
    SM: a run then holds more unvisited vertices than the 4096-entry queue,
    which is filled and drained in windows.  Depths bit-exact, parents a
    valid BFS tree."""
    csr, g = rmat21
    for records in (0, 2):
        eng = S.Engine(g, use_graph=use_graph, direction=S.DIR_PULL, ctas_per_sm=1, pull_gather_ratio=1,
                       pull_runs=1, pull_records=records)
        for src in G.sources(csr, 2, 69) + [int(np.argmax(csr.degree()))]:
            depth, parent, st = eng.bfs(src, parents=True)
            _same(csr, src, depth)
            assert st.pull_levels == st.levels - 1
            rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
            assert rc == 0, f"invalid BFS tree (code {rc} at {bad})"
        eng.close()


def test_rmat21_msbfs_64(rmat21):
    csr, g = rmat21
    eng = S.Engine(g)
    srcs = G.sources(csr, 64, 62)
    depth, st = eng.msbfs(srcs)
    for i, s in enumerate(srcs):
        _same(csr, s, depth[i])
    eng.close()


def test_rmat21_out_of_core(rmat21):
    csr, g = rmat21
    eng = S.Engine(g, pool_bytes=100 * g.pagesize * 4)  # 100 slots for ~600 pages
    for i, src in enumerate(G.sources(csr, 3, 63)):
        if i == 1:
            eng.evict_all()
        depth, _, st = eng.bfs(src)
        _same(csr, src, depth)
        assert st.page_faults > 0 or st.zc_bytes > 0
    eng.close()


def test_rmat22_reference_pages():
    csr = S.Csr.rmat(22, 16, seed=G.SEED + 64, scramble=True)
    g = S.PagedGraph.from_csr(csr)
    eng = S.Engine(g)
    for src in G.sources(csr, 3, 64):
        depth, _, _ = eng.bfs(src)
        _same(csr, src, depth)
    eng.close()


@pytest.mark.parametrize("direction", [S.DIR_ALPHABETA, S.DIR_PULL])
def test_powerlaw2m_directed_in_hbm(powerlaw2m, direction):
    csr, g, gt = powerlaw2m
    eng = S.Engine(g, gt, direction=direction)
    for src in G.sources(csr, 3, 65):
        depth, parent, st = eng.bfs(src, parents=True)
        _same(csr, src, depth)
        rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
        assert rc == 0, f"invalid BFS tree (code {rc} at {bad})"
    eng.close()


def test_powerlaw2m_directed_out_of_core(powerlaw2m):
    csr, g, gt = powerlaw2m
    total = g.npages + gt.npages
    eng = S.Engine(g, gt, pool_bytes=(total // 4) * g.pagesize * 4)
    srcs = G.sources(csr, 3, 66)
    for i, src in enumerate(srcs):
        if i == 1:
            eng.evict_all()
        depth, _, st = eng.bfs(src)
        _same(csr, src, depth)
    # the multi-source traversal through the same pager
    depth, st = eng.msbfs(srcs + G.sources(csr, 61, 67))
    for i, s in enumerate(srcs):
        _same(csr, s, depth[i])
    eng.close()
