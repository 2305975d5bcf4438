"""The learned scheduler against the method without it (alpha/beta + demand
paging), out of core, on held-out sources.  The page link is modelled slow
(page_ms per page fetched) so that, as at full scale, page traffic and not
kernel time dominates; the gain is measured in fetched pages and in that
modelled time.  Depths must stay bit-exact either way."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from scaph_b200 import scheduler
from tests import graphs as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    csr = S.Csr.powerlaw(60000, 900000, 1.9, 3000, seed=G.SEED + 60)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 13)
    gt = S.PagedGraph.from_csr(csr.transpose(), pagesize_words=1 << 13)
    srcs = G.sources(csr, 24, 60)
    return csr, g, gt, srcs[:16], srcs[16:]


def test_traces_and_labels(setup):
    csr, g, gt, train, _ = setup
    tr = scheduler.collect(g, gt, train[:2])
    for t in tr:
        assert t.feats.shape[1] == scheduler.G + g.npages
        assert np.all(t.push_ms[1:] > 0) and np.all(t.pull_ms[1:] > 0)
        dirs, rows, best, ab = scheduler.label(t, 40, 0.5, g.V, g.npages, gt.npages, False)
        assert best <= ab + 1e-9 and dirs[0] == 0 and rows.shape == t.feats.shape


def test_learned_scheduler_beats_alpha_beta_out_of_core(setup):
    csr, g, gt, train, held = setup
    total = g.npages + gt.npages
    nslots = int(0.5 * total)
    pool = nslots * g.pagesize * 4
    page_ms = 0.5
    traces = scheduler.collect(g, gt, train)
    net, info = scheduler.train(traces, g, gt, nslots, page_ms, epochs=300)
    assert info["loss"] < info["loss0"] and info["direction_accuracy"] > 0.8, info
    link_gbs = g.pagesize * 4 / (page_ms * 1e-3) / 1e9  # the modelled link
    plain = scheduler.evaluate(g, gt, held, None, pool)
    learned = scheduler.evaluate(g, gt, held, net, pool, link_gbs=link_gbs)
    for s, a, b in zip(held, plain["depths"], learned["depths"]):
        ref = O.bfs(csr.idx, csr.ngh, s)
        assert np.array_equal(a, ref) and np.array_equal(b, ref)
    cost_plain = plain["ms"] + plain["page_faults"] * page_ms
    cost_learned = learned["ms"] + learned["page_faults"] * page_ms
    print(f"\nalpha/beta: {plain['page_faults']} pages, modelled {cost_plain:.1f} ms; "
          f"learned: {learned['page_faults']} pages (+{learned['prefetched']} prefetched), "
          f"modelled {cost_learned:.1f} ms; training {info}")
    # the traversal waits on demand pages only; prefetches overlap the levels
    assert learned["page_faults"] < plain["page_faults"] // 4
    assert learned["page_faults"] + learned["prefetched"] <= 1.02 * plain["page_faults"]
    assert cost_learned < cost_plain


def test_learned_graph_mode_in_hbm_is_exact_and_matches_host_loop(setup):
    """Resident graph: the learned decision runs on the device inside the
    CUDA-graph traversal; same directions as the host-loop learned engine."""
    csr, g, gt, train, held = setup
    traces = scheduler.collect(g, gt, train[:6])
    net, _ = scheduler.train(traces, g, gt, 64, 0.5, epochs=100)
    eg = S.Engine(g, gt, direction=S.DIR_LEARNED)
    eg.set_scheduler(net)
    eh = S.Engine(g, gt, direction=S.DIR_LEARNED, use_graph=2)
    eh.set_scheduler(net)
    for s in held[:4]:
        dg, _, _ = eg.bfs(s)
        dh, _, _ = eh.bfs(s)
        ref = O.bfs(csr.idx, csr.ngh, s)
        assert np.array_equal(dg, ref) and np.array_equal(dh, ref)
        assert [t["direction"] for t in eg.trace()] == [t["direction"] for t in eh.trace()]
    eg.close()
    eh.close()


def test_learned_multi_source_out_of_core(setup):
    """The network inside the multi-source loop, out of core: the feature
    rows it sees (one per level, the union of the batch's frontiers), the
    in-pages prefetched ahead of the pull levels, and depths still
    bit-exact."""
    csr, g, gt, train, held = setup
    total = g.npages + gt.npages
    pool = int(0.6 * total) * g.pagesize * 4
    rows = scheduler.collect_ms(g, gt, [train[:8], train[8:16]])
    assert all(r.shape[1] == scheduler.G + g.npages for r in rows)
    traces = scheduler.collect(g, gt, train[:6])
    net, info = scheduler.train(traces, g, gt, int(0.6 * total), 0.5, epochs=100, ms_rows=rows)
    assert info["loss"] < info["loss0"]
    eng = S.Engine(g, gt, pool_bytes=pool, direction=S.DIR_LEARNED, record_features=1)
    eng.set_scheduler(net)
    eng.evict_all()
    depth, st = eng.msbfs(held)
    F = eng.features()
    assert F.shape == (st.levels, scheduler.G + g.npages)
    for i, s in enumerate(held):
        assert np.array_equal(depth[i], O.bfs(csr.idx, csr.ngh, s)), f"row {i}"
    eng.close()


def test_multi_source_prefetch_keeps_depths(setup):
    """A network whose direction logit rates every level pull-worthy: each
    push level prefetches the missing in-pages that hold
    incomplete vertices into free slots; the rows stay exact and equal to
    the engine's without a network, and the prefetch count is reported."""
    csr, g, gt, _, held = setup
    net = S.Mlp(scheduler.G + g.npages, 1 + g.npages, seed=5)
    p = net.params()
    n3 = 64 * (1 + g.npages)
    p[-(1 + g.npages) - n3:-(1 + g.npages)] = 0.0  # W3 = 0
    p[-(1 + g.npages):] = 5.0                      # b3: every logit 5
    net.set_params(p)
    total = g.npages + gt.npages
    eng = S.Engine(g, gt, pool_bytes=int(0.8 * total) * g.pagesize * 4, direction=S.DIR_LEARNED)
    eng.set_scheduler(net)
    eng.evict_all()
    depth, st = eng.msbfs(held)
    assert st.prefetched > 0
    assert st.pull_levels > 0
    for i, s in enumerate(held):
        assert np.array_equal(depth[i], O.bfs(csr.idx, csr.ngh, s)), f"row {i}"
    # the same batch without a network gives the same rows
    plain = S.Engine(g, gt, pool_bytes=int(0.8 * total) * g.pagesize * 4)
    plain.evict_all()
    depth_p, _ = plain.msbfs(held)
    assert np.array_equal(depth, depth_p)
    plain.close()
    eng.close()
