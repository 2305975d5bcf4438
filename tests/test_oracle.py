"""The CPU oracle, pinned against the golden fixtures (themselves confirmed by
the reference's own bfs::check) and, where it was built here, against the
reference code in oracle/_ref."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

GOLD = os.path.join(os.path.dirname(__file__), "golden")
UNR = 0xFFFFFFFF
BFS_FIXTURES = sorted(glob.glob(os.path.join(GOLD, "bfs_*.npz")))
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference tree absent)")


def test_fixtures_present():
    assert len(BFS_FIXTURES) >= 6


@pytest.mark.parametrize("path", BFS_FIXTURES, ids=lambda p: os.path.basename(p))
def test_oracle_matches_golden(path):
    z = np.load(path)
    for i, s in enumerate(z["sources"]):
        s = int(s)
        assert np.array_equal(O.bfs(z["idx"], z["ngh"], s, 63), z["depth63"][i])
        assert np.array_equal(O.bfs(z["idx"], z["ngh"], s, UNR), z["depth"][i])
        assert np.array_equal(O.bfs_omp(z["idx"], z["ngh"], s, UNR, 4), z["depth"][i])


@pytest.mark.parametrize("path", BFS_FIXTURES, ids=lambda p: os.path.basename(p))
def test_paged_walk_matches_golden(path):
    z = np.load(path)
    csr = S.Csr.from_arrays(z["idx"], z["ngh"])
    g = S.PagedGraph.from_csr(csr, pagesize_words=256 if csr.V < 200 else 4096)
    pages = [g.page(p) for p in range(g.npages)]
    for i, s in enumerate(z["sources"]):
        assert np.array_equal(O.bfs_paged(csr.V, g.page_list(), pages, int(s), UNR), z["depth"][i])


@needs_ref
def test_reference_check_agrees_with_oracle():
    """The reference's own bfs::check finds 0 mismatches in the oracle's depths
    and exactly the planted ones otherwise."""
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 50)
    idx32 = csr.idx.astype(np.uint32)
    for s in G.sources(csr, 3, 50):
        d = O.bfs(csr.idx, csr.ngh, s, 63)
        assert O.ref_bfs_check(idx32, csr.ngh, s, d)[0] == 0
        bad = d.copy()
        bad[[1, 7, 99]] ^= 1
        assert O.ref_bfs_check(idx32, csr.ngh, s, bad)[0] == 3


def test_reference_depth_cap_63():
    """Depths >= 63 are unrepresentable in the reference (cond is d > s+1 with
    MAXDEPTH 63): the restatement reproduces that cap."""
    z = np.load(os.path.join(GOLD, "bfs_path100.npz"))
    d = z["depth63"][0]  # from vertex 0 of a 100-path
    assert d[62] == 62 and (d[63:] == 63).all()
    assert (z["depth"][0] == np.arange(100)).all()


def test_validator_accepts_oracle_tree_and_rejects_planted_errors():
    csr = S.Csr.rmat(12, 16, seed=G.SEED + 51)
    s = G.sources(csr, 1, 51)[0]
    d = O.bfs(csr.idx, csr.ngh, s)
    # build a parent array on the CPU: any neighbour one level up
    parent = np.full(csr.V, UNR, np.uint32)
    parent[s] = s
    idx, ngh = csr.idx, csr.ngh
    for v in np.flatnonzero((d != UNR) & (np.arange(csr.V) != s)):
        nb = ngh[idx[v]:idx[v + 1]]
        parent[v] = nb[d[nb] == d[v] - 1][0]
    assert O.validate_tree(idx, ngh, s, d, parent)[0] == 0
    v = int(np.flatnonzero(d == 2)[0])
    p2 = parent.copy()
    p2[v] = s  # depth mismatch (depth[s]+1 != 2)
    assert O.validate_tree(idx, ngh, s, d, p2)[0] == -3
    p3 = parent.copy()
    p3[s] = (s + 1) % csr.V
    assert O.validate_tree(idx, ngh, s, d, p3)[0] == -1
    u = int(np.flatnonzero(d == UNR)[0])
    p4 = parent.copy()
    p4[u] = s
    assert O.validate_tree(idx, ngh, s, d, p4)[0] == -5


def test_page_stats_restatement():
    """get_page_info (src/gpu_engine.cuh:397-441): per-page sum of stat and of stat*(deg+3)."""
    csr = S.Csr.rmat(12, 16, seed=G.SEED + 52)
    g = S.PagedGraph.from_csr(csr, pagesize_words=2048)
    rng = np.random.default_rng(52)
    stat = (rng.random(csr.V) < 0.3).astype(np.uint8)
    deg = csr.degree()
    nodes, datas, tn, td = O.page_stats(g.page_list(), stat, deg)
    for p, (left, right, _, _) in enumerate(g.page_list()):
        sl = slice(int(left), int(right) + 1)
        assert nodes[p] == stat[sl].sum()
        assert datas[p] == (stat[sl].astype(np.int64) * (deg[sl].astype(np.int64) + 3)).sum()
    assert tn == stat.sum() and td == datas.sum()


def _compress_graph():
    meta = json.load(open(os.path.join(GOLD, "chunk_and_compress.json")))["compress_stat"]
    gm = meta["graph"]
    csr = S.Csr.rmat(gm["scale"], 16, seed=gm["seed"])
    return meta, S.PagedGraph.from_csr(csr, pagesize_words=gm["pagesize_words"])


def test_compaction_restatement_matches_golden():
    """compress_stat (src/compress.h:18-40) restated == the reference's output."""
    meta, g = _compress_graph()
    pl = g.page_list()
    for name, rec in meta["pages"].items():
        p = int(name[4:])
        left, right, n, e = (int(x) for x in pl[p])
        stat = np.load(os.path.join(GOLD, f"compress_stat_{name}.npy"))
        active = int(stat[left:right + 1].sum())
        dst, cnt = O.compact_page(g.page(p), stat, left, n, active, out_words=g.pagesize)
        assert cnt == rec["active"]
        assert hashlib.sha256(dst.tobytes()).hexdigest() == rec["sha256"]


@needs_ref
def test_compaction_restatement_matches_reference_live():
    csr = S.Csr.rmat(12, 16, seed=G.SEED + 53)
    g = S.PagedGraph.from_csr(csr, pagesize_words=4096)
    rng = np.random.default_rng(53)
    for p, (left, right, n, e) in enumerate(g.page_list()):
        stat = (rng.random(csr.V) < 0.1 * (p % 5 + 1)).astype(np.uint8)
        active = int(stat[left:right + 1].sum())
        mine, cnt = O.compact_page(g.page(p), stat, int(left), int(n), active, out_words=g.pagesize)
        ref = np.zeros(g.pagesize, np.uint32)
        src = g.page(p).copy()
        rc = O.rlib().ref_compress_stat(O._p(src), O._p(ref), O._p(stat), int(left), int(n), active)
        assert rc == cnt and np.array_equal(mine, ref)


def test_chunk_mask_helpers_match_golden():
    """Best-fit contiguous free-chunk run (src/tools.h:11-64)."""
    rows = json.load(open(os.path.join(GOLD, "chunk_and_compress.json")))["chunk_masks"]
    L = O.olib()
    for r in rows:
        assert L.oracle_max_zero_run(r["mask"]) == r["max"]
        for req, fit in enumerate(r["fit"], start=1):
            assert L.oracle_fit_zero_run(r["mask"], req) == fit, (hex(r["mask"]), req)


@needs_ref
def test_set_run_matches_reference():
    L = O.olib()
    rng = np.random.default_rng(54)
    for _ in range(200):
        m = int(rng.integers(0, 2**31))
        off = int(rng.integers(0, 32))
        n = int(rng.integers(0, 33 - off))
        for val in (0, 1):
            ref = O.rlib().ref_set_run(m, off, n, val) & 0xFFFFFFFF
            assert L.oracle_set_run(m, off, n, val) == ref


@pytest.mark.parametrize("scale,ef,seed,scramble", [(8, 16, 1, True), (12, 16, 0x5CA90001, True),
                                                    (14, 8, 7, False), (17, 32, 0x5CA90003, True)])
def test_oracle_rmat_generator_equals_the_library_generator(scale, ef, seed, scramble):
    """bench.py's reference arm builds its graph with the oracle's generator
    (no product library in that process): it must give the same CSR."""
    idx, ngh = O.gen_rmat(scale, ef, 0.57, 0.19, 0.19, seed, scramble)
    csr = S.Csr.rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed, scramble=scramble)
    assert np.array_equal(idx, csr.idx)
    assert np.array_equal(ngh, csr.ngh)


def test_reference_arm_workload_equals_ours():
    """Same graph and same sources in both bench arms (small scale)."""
    import bench
    from scaph_b200 import workloads

    idx, ngh, srcs = bench.rmat24_for_reference(14, 16)
    csr, srcs2 = workloads.config2(14, 16)
    assert srcs == srcs2
    assert np.array_equal(idx, csr.idx) and np.array_equal(ngh, csr.ngh)
    assert bench.config_dict(len(idx) - 1, len(ngh), 14, 16) == bench.config_dict(csr.V, csr.E, 14, len(srcs2))
