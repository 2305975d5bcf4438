"""The learned scheduler's training labels on the CPU: on synthetic traces,
scheduler.label's cheapest direction sequence - the better of alpha/beta's
own sequence and every push -> pull -> push shape starting with push -
equals a brute force, resident and with a cold pool large enough never to
evict; alpha/beta's cost is its own sequence's; the label never costs more
than alpha/beta."""
import itertools

import numpy as np
import pytest

from scaph_b200 import scheduler as SC

V = 100_000


def synthetic_trace(rng, L, n_out, n_in):
    nf = rng.integers(1, V // 4, L).astype(np.float64)
    nf[0] = 1
    mf = nf * rng.uniform(1, 40, L)
    mu = np.maximum(1.0, np.cumsum(mf[::-1])[::-1] * rng.uniform(1, 3))
    out_need = [rng.choice(n_out, rng.integers(0, n_out + 1), replace=False) for _ in range(L)]
    in_need = [rng.choice(n_in, rng.integers(0, n_in + 1), replace=False) for _ in range(L)]
    return SC.Trace(
        src=0,
        feats=np.zeros((L, SC.G + n_out), np.float32),
        push_ms=rng.uniform(0.01, 1.0, L),
        pull_ms=rng.uniform(0.01, 1.0, L),
        nf=nf, mf=mf, mu=mu,
        out_need=out_need, in_need=in_need,
        out_datas=[np.full(len(p), 1000) for p in out_need], in_datas=[np.full(len(p), 1000) for p in in_need],
        next_active=np.zeros((L, n_out), np.float32))


def brute(tr, page_ms, gin):
    L = len(tr.push_ms)
    best = None
    for tail in itertools.product((0, 1), repeat=L - 1):
        seq = (0,) + tail
        runs = [k for k, _ in itertools.groupby(seq)]
        if runs not in ([0], [0, 1], [0, 1, 0]):
            continue
        seen, total = set(), 0.0
        for lvl, d in enumerate(seq):
            total += tr.push_ms[lvl] if d == 0 else tr.pull_ms[lvl]
            need = {(0, int(p)) for p in tr.out_need[lvl]} if d == 0 else {(gin, int(p)) for p in tr.in_need[lvl]}
            total += page_ms * len(need - seen)  # a cold pool that never evicts fetches a page once
            seen |= need
        best = total if best is None else min(best, total)
    return best


@pytest.mark.parametrize("seed", range(6))
def test_resident_label_is_the_brute_force_optimum(seed):
    rng = np.random.default_rng(seed)
    L = int(rng.integers(2, 9))
    tr = synthetic_trace(rng, L, 6, 6)
    dirs, rows, best, ab = SC.label(tr, 4, 1.0, V, 6, 6, False, resident=True)
    assert dirs[0] == 0 and rows.shape == tr.feats.shape
    assert best == pytest.approx(min(brute(tr, 0.0, 1), ab))
    assert best <= ab + 1e-9
    # alpha/beta's cost is its own sequence's kernel time
    seq = [0]
    for lvl in range(1, L):
        seq.append(SC.alpha_beta(seq[-1], tr.nf[lvl], tr.nf[lvl - 1], tr.mf[lvl], tr.mu[lvl], V))
    assert ab == pytest.approx(sum(tr.push_ms[i] if d == 0 else tr.pull_ms[i] for i, d in enumerate(seq)))
    # the label's cost is the cost of the sequence it returns
    assert best == pytest.approx(sum(tr.push_ms[i] if d == 0 else tr.pull_ms[i] for i, d in enumerate(dirs)))


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("symmetric", [False, True])
def test_cold_pool_label_counts_each_page_once(seed, symmetric):
    rng = np.random.default_rng(100 + seed)
    L = int(rng.integers(2, 8))
    n = 5
    tr = synthetic_trace(rng, L, n, n)
    page_ms = float(rng.uniform(0.05, 0.5))
    gin = 0 if symmetric else 1
    dirs, _, best, ab = SC.label(tr, 2 * n, page_ms, V, n, n, symmetric)
    assert dirs[0] == 0
    assert best == pytest.approx(min(brute(tr, page_ms, gin), ab))
    assert best <= ab + 1e-9


def test_sequences_are_the_push_pull_push_shapes():
    for L in range(1, 7):
        seqs = [tuple(s) for s in SC.sequences(L)]  # may repeat a sequence (harmless)
        expected = {(0,) + t for t in itertools.product((0, 1), repeat=L - 1)
                    if [k for k, _ in itertools.groupby((0,) + t)] in ([0], [0, 1], [0, 1, 0])}
        assert set(seqs) == expected
