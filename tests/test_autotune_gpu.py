"""Engine tunables and the autotuner: every tunable changes the schedule
only (depths bit-exact with the oracle under each setting), bad values are
rejected, and the coordinate search returns a setting that reproduces the
default's depths."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from scaph_b200 import autotune
from tests import graphs as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat15():
    csr = S.Csr.rmat(15, 16, seed=G.SEED + 80)
    return csr, S.PagedGraph.from_csr(csr, pagesize_words=1 << 15)


@pytest.mark.parametrize("kw", [dict(giant_edges=128), dict(giant_edges=8192), dict(pull_gather_ratio=1),
                                dict(pull_gather_ratio=100000), dict(ctas_per_sm=1, block_size=512),
                                dict(alpha=2.0, beta=200.0), dict(push_defer_edges=1),
                                dict(push_defer_edges=1, giant_edges=256, alpha=0.01), dict(pull_warp=1),
                                dict(pull_warp=1, alpha=0.01, beta=0.001), dict(pull_warp=1, block_size=128),
                                dict(pull_records=1), dict(pull_records=2), dict(pull_records=1, pull_warp=1),
                                dict(pull_warp=2, pull_records=1), dict(pull_warp=2, pull_records=1, alpha=0.01, beta=0.001),
                                dict(pull_warp=2, pull_records=1, block_size=512), dict(pull_warp=3, pull_records=1),
                                dict(push_defer_edges=-1), dict(pull_rows=2), dict(pull_rows=1, pull_records=2),
                                dict(pull_rows=1, pull_records=2, alpha=0.01, beta=0.001),
                                dict(pull_rows=1, pull_records=2, pull_gather_ratio=1), dict(push_sparse_ratio=-1),
                                dict(push_sparse_ratio=1, alpha=0.01), dict(push_sparse_ratio=1, alpha=0.01, block_size=128),
                                dict(push_sparse_ratio=1, alpha=0.01, block_size=512, push_defer_edges=1),
                                dict(pull_runs=2), dict(pull_runs=2, pull_gather_ratio=1),
                                dict(pull_runs=1, pull_gather_ratio=1), dict(pull_runs=1, pull_gather_ratio=1, block_size=512),
                                dict(pull_runs=1, pull_gather_ratio=1, pull_records=2, pull_rows=1)])
def test_tunables_keep_depths(rmat15, kw):
    """push_defer_edges=1 defers the claims of every push level (neighbours
    OR-ed into the next frontier, depths written by the finalize pass);
    with alpha 0.01 every level pushes (the switch to pull needs
    more than 100 times the unvisited edges in the frontier)."""
    csr, g = rmat15
    for use_graph in (0, 2):
        eng = S.Engine(g, use_graph=use_graph)
        eng.tune(**kw)
        for src in G.sources(csr, 2, 80) + [int(np.argmax(csr.degree()))]:
            d, _, _ = eng.bfs(src)
            assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src)), (kw, use_graph, src)
        eng.close()


@pytest.mark.parametrize("kw", [dict(ms_compact_l2_div=1, ms_compact_min_deg=1),
                                dict(ms_compact_l2_div=1000, ms_compact_min_deg=1000)])
def test_ms_tunables_keep_depths(rmat15, kw):
    csr, g = rmat15
    eng = S.Engine(g)
    eng.tune(**kw)
    srcs = G.sources(csr, 40, 81)
    d, _ = eng.msbfs(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(d[i], O.bfs(csr.idx, csr.ngh, s))
    eng.close()


def test_tune_rejects_bad_values(rmat15):
    _, g = rmat15
    eng = S.Engine(g)
    for kw in (dict(giant_edges=64), dict(giant_edges=1 << 20), dict(block_size=384)):
        with pytest.raises(S.ScaphError) as ex:
            eng.tune(**kw)
        assert ex.value.code == S.EINVAL
        eng.tune(giant_edges=1024, block_size=256)
    with pytest.raises(S.ScaphError):
        eng.tune(no_such_knob=1)
    eng.close()


def test_autotune_engine_single_and_multi(rmat15):
    import torch

    csr, g = rmat15
    eng = S.Engine(g)
    srcs = G.sources(csr, 4, 82)
    buf = torch.empty(len(srcs) * csr.V, dtype=torch.int32, device="cuda")
    r = autotune.tune_engine(eng, srcs, buf.data_ptr(), repeats=2)
    assert r["tried"] > 10 and r["ms"] <= r["default_ms"]
    assert set(r["params"]) == set(S.Engine.TUNABLES)
    for s in srcs:
        d, _, _ = eng.bfs(s)
        assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, s))
    r = autotune.tune_engine(eng, srcs, buf.data_ptr(), multi=True, repeats=2)
    assert r["ms"] <= r["default_ms"]
    eng.close()


def test_deferred_push_with_parents_falls_back_to_claims(rmat15):
    """Parents need a claim winner: with parents requested the deferred path
    is not taken, and the tree is valid."""
    csr, g = rmat15
    eng = S.Engine(g, push_defer_edges=1)
    src = G.sources(csr, 1, 83)[0]
    d, p, _ = eng.bfs(src, parents=True)
    assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src))
    rc, bad = O.validate_tree(csr.idx, csr.ngh, src, d, p)
    assert rc == 0, (rc, bad)
    eng.close()
