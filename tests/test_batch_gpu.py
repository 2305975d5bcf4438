"""Mixed query batches (scaph_batch_*): many single-source queries over
graphs of uneven size in one CUDA-graph launch, bit-exact with the CPU
oracle on every query; the autotuner's parameters never change depths."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from scaph_b200 import autotune
from tests import graphs as G

pytestmark = pytest.mark.gpu


def check_rows(graphs, queries, rows, unreached=S.UNREACHED):
    for (g, s), row in zip(queries, rows):
        csr = graphs[g]
        ref = O.bfs(csr.idx, csr.ngh, s, unreached=unreached)
        assert np.array_equal(row, ref), (g, s, int(np.flatnonzero(row != ref)[0]))


@pytest.fixture(scope="module")
def mixed():
    graphs = [S.Csr.rmat(sc, ef, seed=G.SEED + 100 + i) for i, (sc, ef) in
              enumerate([(8, 8), (12, 16), (10, 32), (13, 8), (9, 12), (11, 24)])]
    graphs.append(G.path(300))      # 299 levels: more than the first launch's depth planes
    graphs.append(G.star(50, 7))
    rng = np.random.default_rng(5)
    queries = []
    for _ in range(60):
        g = int(rng.integers(0, len(graphs)))
        queries.append((g, int(rng.integers(0, graphs[g].V))))
    queries += [(6, 0), (6, 299), (7, 7), (1, queries[1][1] if queries[1][0] == 1 else 0)]
    queries.append(queries[0])      # a repeated query
    return graphs, queries


def test_batch_matches_oracle_every_query(mixed):
    graphs, queries = mixed
    b = S.Batch(graphs, pagesize_words=1 << 12)
    rows, st = b.run(queries)
    assert st.launches == 1 and st.levels >= 299
    check_rows(graphs, queries, rows)
    # run again (graph reused) with the queries shuffled
    perm = np.random.default_rng(1).permutation(len(queries))
    q2 = [queries[i] for i in perm]
    rows2, _ = b.run(q2)
    check_rows(graphs, q2, rows2)
    b.close()


def test_batch_two_mask_words_and_reference_sentinel(mixed):
    graphs, _ = mixed
    rng = np.random.default_rng(9)
    queries = [(1, int(v)) for v in rng.integers(0, graphs[1].V, 100)] + [(3, 5), (0, 1)]
    b = S.Batch(graphs[:4], pagesize_words=1 << 12, unreached=63)
    rows, st = b.run(queries)
    check_rows(graphs, queries, rows, unreached=63)
    with pytest.raises(S.ScaphError) as ei:
        b.run([(1, 0)] * 129)
    assert ei.value.code == S.EINVAL
    with pytest.raises(S.ScaphError):
        b.run([(9, 0)])
    b.close()


def test_batch_directed_graphs_with_transposes():
    graphs = [S.Csr.powerlaw(3000 + 1000 * i, 20000 + 5000 * i, 1.9, 500, seed=G.SEED + 110 + i) for i in range(4)]
    trans = [g.transpose() for g in graphs]
    rng = np.random.default_rng(11)
    queries = [(int(g), int(rng.integers(0, graphs[g].V))) for g in rng.integers(0, 4, 40)]
    b = S.Batch(graphs, trans, pagesize_words=1 << 12)
    rows, st = b.run(queries)
    check_rows(graphs, queries, rows)
    assert st.pull_levels + st.push_levels == st.levels
    b.close()


def test_every_parameter_choice_gives_the_same_depths(mixed):
    graphs, queries = mixed
    b = S.Batch(graphs[:6], pagesize_words=1 << 12)
    q = [x for x in queries if x[0] < 6]
    ref, _ = b.run(q)
    check_rows(graphs, q, ref)
    for (blk, c) in autotune.SHAPES:
        for a, bt in ((14.0, 24.0), (7.0, 96.0), (28.0, 12.0)):
            b.set_params(blk, c, a, bt)
            rows, _ = b.run(q)
            for r0, r1 in zip(ref, rows):
                assert np.array_equal(r0, r1), (blk, c, a, bt)
    b.close()


def test_autotuner_picks_and_caches(mixed, tmp_path):
    import torch

    graphs, queries = mixed
    b = S.Batch(graphs[:6], pagesize_words=1 << 12)
    q = [x for x in queries if x[0] < 6]
    buf = torch.empty(b.out_words(q), dtype=torch.int32, device="cuda")
    cache = str(tmp_path / "tune.json")
    r1 = autotune.tune_batch(b, q, buf.data_ptr(), repeats=1, cache=cache)
    assert not r1["cached"] and r1["tried"] > 10 and r1["ms"] <= r1["default_ms"]
    b2 = S.Batch(graphs[:6], pagesize_words=1 << 12)
    r2 = autotune.tune_batch(b2, q, buf.data_ptr(), cache=cache)
    assert r2["cached"] and b2.params == pytest.approx(r1["params"])
    rows, _ = b2.run(q)
    check_rows(graphs, q, rows)
    b.close()
    b2.close()
