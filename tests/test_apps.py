"""App-hook layer on the CPU: the oracle of the reference's vertex programs
(BFS / SSSP / WCC hooks) pinned against independent algorithms and against a
restatement of the reference's own WCC check, the paged->flat CSR read-back,
and the reference's unmodified applications compiling against
include/scaph/compat."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_APP = os.path.join(O.REFERENCE_DIR, "app")
FAR_BFS = 63           # MAXDEPTH of app/bfs.cu:18
FAR_SSSP = 0x7FFFFFFF  # MAXPATH of app/sssp.cu:11


def weighted(csr: S.Csr, seed: int, wmax: int = 100) -> S.Csr:
    rng = np.random.default_rng(seed)
    w = rng.integers(1, wmax + 1, csr.E).astype(np.uint32)
    return S.Csr.from_arrays(csr.idx, csr.ngh, w)


def single_source(V, src, far):
    value = np.full(V, far, np.uint32)
    value[src] = 0
    active = np.zeros(V, np.uint8)
    active[src] = 1
    return value, active


def ref_wcc_check(idx, ngh):
    """The CPU labelling of wcc::check (app/wcc.cu:59-83), loop for loop:
    sweep all vertices until a sweep lowers nothing."""
    V = len(idx) - 1
    value = list(range(V))
    active = V
    while active > 0:
        active = 0
        for v in range(V):
            for e in range(int(idx[v]), int(idx[v + 1])):
                u = int(ngh[e])
                if value[v] < value[u]:
                    value[u] = value[v]
                    active += 1
    return np.array(value, np.uint32)


@pytest.mark.parametrize("symmetric", [True, False])
def test_bfs_hooks_fixpoint_is_capped_level_bfs(symmetric):
    csr = G.random_graph(3000, 9000, G.SEED + 70, symmetric=symmetric)
    for src in G.sources(csr, 3, 71):
        for far in (FAR_BFS, 5, 0xFFFFFFFF):
            value, active = single_source(csr.V, src, far)
            got = O.hook_fixpoint(csr.idx, csr.ngh, "bfs", value, active)
            ref = O.bfs(csr.idx, csr.ngh, src, unreached=far)
            assert np.array_equal(got, np.minimum(ref, far))


def test_sssp_hooks_fixpoint_is_dijkstra():
    csr = weighted(G.random_graph(4000, 20000, G.SEED + 72, symmetric=False), 73)
    for src in G.sources(csr, 3, 74):
        value, active = single_source(csr.V, src, FAR_SSSP)
        got = O.hook_fixpoint(csr.idx, csr.ngh, "sssp", value, active, wgh=csr.wgh)
        assert np.array_equal(got, O.sssp_dijkstra(csr.idx, csr.ngh, csr.wgh, src, FAR_SSSP))
        # a tight cap: everything at or past it stays at the cap
        value, active = single_source(csr.V, src, 150)
        got = O.hook_fixpoint(csr.idx, csr.ngh, "sssp", value, active, wgh=csr.wgh)
        assert np.array_equal(got, O.sssp_dijkstra(csr.idx, csr.ngh, csr.wgh, src, 150))


@pytest.mark.parametrize("symmetric", [True, False])
def test_wcc_hooks_fixpoint_is_min_reaching_id(symmetric):
    csr = G.random_graph(5000, 6000, G.SEED + 75, symmetric=symmetric)
    V = csr.V
    got = O.hook_fixpoint(csr.idx, csr.ngh, "wcc", np.arange(V, dtype=np.uint32), np.ones(V, np.uint8))
    assert np.array_equal(got, O.min_reaching_id(csr.idx, csr.ngh))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_wcc_oracle_matches_the_reference_check_loop(seed):
    csr = G.random_graph(120, 150, G.SEED + 76 + seed, symmetric=bool(seed % 2))
    V = csr.V
    got = O.hook_fixpoint(csr.idx, csr.ngh, "wcc", np.arange(V, dtype=np.uint32), np.ones(V, np.uint8))
    assert np.array_equal(got, ref_wcc_check(csr.idx, csr.ngh))


def test_graph_to_csr_reads_back_the_pages():
    csr = G.random_graph(2000, 12000, G.SEED + 80, symmetric=False)
    for w in (False, True):
        src = weighted(csr, 81) if w else csr
        g = S.PagedGraph.from_csr(src, 1 << 10, weighted=w)
        assert g.npages > 3
        back = g.to_csr()
        assert np.array_equal(back.idx, src.idx) and np.array_equal(back.ngh, src.ngh)
        if w:
            assert np.array_equal(back.wgh, src.wgh)
        else:
            assert back.wgh is None


def test_csr_symmetric():
    assert S.Csr.rmat(10, 8, seed=3).symmetric()
    assert G.random_graph(500, 2000, G.SEED + 82, symmetric=True).symmetric()
    assert not G.random_graph(500, 2000, G.SEED + 82, symmetric=False).symmetric()
    assert G.path(10).symmetric()
    one_way = G.csr_from_edges(3, [0], [1])
    assert not one_way.symmetric()


def test_example_apps_are_built():
    for name in ("bfs", "sssp", "wcc"):
        p = os.path.join(ROOT, "scaph_b200", "apps", "_build", name)
        assert os.access(p, os.X_OK), f"{p} missing: run __graft_entry__.build()"


@pytest.mark.skipif(not os.path.isdir(REF_APP) or shutil.which("nvcc") is None,
                    reason="reference application sources or nvcc not available")
def test_reference_apps_build_unchanged_against_compat(tmp_path):
    """app/bfs.cu, app/sssp.cu and app/wcc.cu, as they are, compile and
    link against scaph/compat/app.cuh + libscaph."""
    out = tmp_path / "apps"
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "scaph_b200", "apps"), "ref",
                        f"REF_APP_DIR={REF_APP}", f"OUT={out}", "-j3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    for name in ("bfs", "sssp", "wcc"):
        assert os.access(out / "ref" / name, os.X_OK)


def test_pagerank_oracle_against_the_google_matrix():
    """The float64 PageRank oracle equals the power iteration of the explicit
    Google matrix (dangling vertices spread uniformly) on a small directed
    graph, and its ranks sum to 1."""
    csr = G.random_graph(60, 200, seed=11, symmetric=False)
    V = csr.V
    M = np.zeros((V, V))
    deg = csr.degree()
    for u in range(V):
        nb = csr.ngh[csr.idx[u]:csr.idx[u + 1]]
        if len(nb):
            M[nb, u] += 1.0 / len(nb)
        else:
            M[:, u] = 1.0 / V
    d = 0.85
    Gm = d * M + (1 - d) / V
    r = np.full(V, 1.0 / V)
    for _ in range(30):
        r = Gm @ r
    got = O.pagerank(csr.idx, csr.ngh, 30, d)
    assert np.allclose(got, r, rtol=1e-12, atol=1e-15)
    assert abs(got.sum() - 1.0) < 1e-12
    assert (deg == 0).any()
