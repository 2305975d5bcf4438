"""Multi-source BFS: every row of the batched result is bit-exact with the
oracle's single-source BFS from that source."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu


def check_batch(csr, eng, srcs, unreached=S.UNREACHED):
    depth, st = eng.msbfs(srcs)
    for i, s in enumerate(srcs):
        ref = O.bfs(csr.idx, csr.ngh, int(s), unreached)
        bad = np.flatnonzero(depth[i] != ref)
        assert bad.size == 0, f"row {i} (src {s}): {bad.size} mismatches, v={bad[0]} gpu={depth[i][bad[0]]} " \
                              f"cpu={ref[bad[0]]}"
    return depth, st


@pytest.mark.parametrize("direction", [S.DIR_ALPHABETA, S.DIR_PUSH, S.DIR_PULL])
def test_msbfs_64_sources_rmat(direction):
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 20)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    eng = S.Engine(g, direction=direction)
    check_batch(csr, eng, G.sources(csr, 64, 20))
    eng.close()


def test_msbfs_128_sources_two_words_and_repeat():
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 21)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 13)
    eng = S.Engine(g)
    srcs = G.sources(csr, 120, 21) + [0, 0, 5, 5, 7, 9, 11, 13]  # duplicates and isolated ids too
    check_batch(csr, eng, srcs)
    # a second, smaller batch on the same engine reuses the state
    check_batch(csr, eng, srcs[:3])
    check_batch(csr, eng, srcs[:70])
    eng.close()


def test_msbfs_single_source_and_cap():
    csr = G.path(200)
    g = S.PagedGraph.from_csr(csr, pagesize_words=256)
    eng = S.Engine(g)
    check_batch(csr, eng, [0])
    check_batch(csr, eng, [0, 199, 100])
    eng.close()
    eng = S.Engine(g, unreached=S.REF_UNREACHED)
    d, _ = check_batch(csr, eng, [0, 199, 100], S.REF_UNREACHED)
    assert d[0].max() == 63
    eng.close()


@pytest.mark.parametrize("direction", [S.DIR_ALPHABETA, S.DIR_PULL])
def test_msbfs_directed_with_transpose(direction):
    csr = S.Csr.powerlaw(20000, 250000, 1.9, 2000, seed=G.SEED + 22)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 14)
    gt = S.PagedGraph.from_csr(csr.transpose(), pagesize_words=1 << 14)
    eng = S.Engine(g, gt, direction=direction)
    check_batch(csr, eng, G.sources(csr, 64, 22))
    eng.close()


def test_msbfs_hub_giant_chunks():
    csr = G.star(9000, center=5)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 15)
    eng = S.Engine(g, direction=S.DIR_PUSH)
    check_batch(csr, eng, [5, 6, 7, 8000])
    eng.close()


def test_msbfs_matches_single_source_engine_and_trace():
    csr = S.Csr.rmat(15, 16, seed=G.SEED + 23)
    g = S.PagedGraph.from_csr(csr)
    eng = S.Engine(g)
    srcs = G.sources(csr, 32, 23)
    d, st = eng.msbfs(srcs)
    for i in (0, 13, 31):
        single, _, _ = eng.bfs(srcs[i])
        assert np.array_equal(single, d[i])
    tr = eng.msbfs_trace()
    assert len(tr) == st.levels and st.reached == int((d != S.UNREACHED).sum())
    eng.close()


@pytest.mark.parametrize("direction", [S.DIR_ALPHABETA, S.DIR_PUSH, S.DIR_PULL, S.DIR_LEARNED])
def test_msbfs_out_of_core(direction):
    """Pool of a third of the out+in pages: the multi-source levels run on
    page batches (resident, zero-copy, demand copies); depths still exact.
    DIR_LEARNED adds the out-of-core transfer rule to alpha/beta."""
    csr = S.Csr.powerlaw(30000, 400000, 1.9, 3000, seed=G.SEED + 23)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 12)
    gt = S.PagedGraph.from_csr(csr.transpose(), pagesize_words=1 << 12)
    total = g.npages + gt.npages
    pool = (total // 3) * g.pagesize * 4
    eng = S.Engine(g, gt, pool_bytes=pool, direction=direction, compact_threshold=2)
    srcs = G.sources(csr, 100, 23)
    for cold in (True, False):
        if cold:
            eng.evict_all()
        _, st = check_batch(csr, eng, srcs)
        assert st.h2d_bytes + st.zc_bytes > 0
        assert st.push_levels + st.pull_levels == st.levels
    tr = eng.msbfs_trace()
    assert sum(t["h2d_bytes"] for t in tr) > 0 or not cold
    eng.close()


def test_msbfs_out_of_core_symmetric_64():
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 24)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 13)
    eng = S.Engine(g, pool_bytes=(g.npages // 2) * g.pagesize * 4)
    check_batch(csr, eng, G.sources(csr, 64, 24))
    eng.close()


@pytest.mark.parametrize("pool", [0, 1], ids=["resident", "out_of_core"])
def test_msbfs_all_vertices_in_frontier(pool):
    """A small web-like graph (blocks of 4096 ids, every vertex reachable)
    with 128 sources: the union frontier holds every vertex for some levels,
    where the pull reads neighbours' masks without their frontier bits.
    Every row bit-exact, resident and through the pager."""
    from scaph_b200 import workloads

    csr, tcsr = workloads.config5(V=200_000, E=7_000_000)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 20)
    gt = S.PagedGraph.from_csr(tcsr, pagesize_words=1 << 20)
    total = g.npages + gt.npages
    eng = S.Engine(g, gt, pool_bytes=(total // 2) * g.pagesize * 4 if pool else 0)
    srcs = G.sources(csr, 128, 90)
    depth, st = eng.msbfs(srcs)
    tr = eng.msbfs_trace()
    assert any(t["frontier"] == csr.V and t["direction"] == 1 for t in tr), [t["frontier"] for t in tr]
    for i in range(0, 128, 9):
        ref = O.bfs(csr.idx, csr.ngh, int(srcs[i]))
        assert np.array_equal(depth[i], ref), f"row {i}"
    eng.close()
