"""The engine autotuner's search and adoption rules on the CPU, against a
fake engine whose device times are a function of its tunables: a setting
that is clearly faster is adopted (and confirmed by interleaved reruns);
gains inside the default's own run-to-run spread leave the defaults; a
setting that changes the depths is refused and the defaults restored; the
multi-source search covers its own axes; the mixed-batch tuner finds the
best launch shape and reuses it from its cache for a batch of the same
shape."""
import numpy as np
import pytest

import scaph_b200 as S
from scaph_b200 import autotune


class _Stats:
    def __init__(self, ms):
        self.ms = ms


class FakeEngine:
    """Times: base_ms, scaled by `factors[(name, value)]` for each tunable
    set to a listed value, plus uniform noise of +-noise (relative)."""

    def __init__(self, factors=None, noise=0.0, bad=None, seed=0):
        self.p = dict(S.Engine._TUNABLE_DEFAULTS)
        self.p.update({"alpha": 14.0, "beta": 96.0, "block_size": 256, "ctas_per_sm": 0, "pull_records": 0})
        self.factors = factors or {}
        self.noise = noise
        self.bad = bad  # (name, value) whose setting changes the depths
        self.rng = np.random.default_rng(seed)
        self.tune_calls = 0

    def tunables(self):
        return dict(self.p)

    def tune(self, **kw):
        for k in kw:
            assert k in S.Engine.TUNABLES, k
        self.p.update(kw)
        self.tune_calls += 1

    def _ms(self):
        f = 1.0
        for (name, value), x in self.factors.items():
            if self.p.get(name) == value:
                f *= x
        return 1.0 * f * (1.0 + self.noise * (2 * self.rng.random() - 1))

    def _depth(self, s):
        d = np.arange(64, dtype=np.uint32) + np.uint32(s)
        if self.bad and self.p.get(self.bad[0]) == self.bad[1]:
            d[3] += 1
        return d

    def bfs_device(self, s, ptr):
        return _Stats(self._ms())

    def bfs(self, s):
        return self._depth(s), None, _Stats(self._ms())

    def msbfs_device(self, srcs, ptr):
        return _Stats(self._ms())

    def msbfs(self, srcs):
        return np.stack([self._depth(s) for s in srcs]), _Stats(self._ms())


def test_clear_gain_is_adopted_and_confirmed():
    eng = FakeEngine(factors={("pull_warp", 3): 0.8}, noise=0.001)
    r = autotune.tune_engine(eng, [1, 2, 3], 0)
    assert r["adopted"] == "tuned" and r["gain_beyond_noise"]
    assert r["params"]["pull_warp"] == 3
    assert eng.tunables()["pull_warp"] == 3  # the adopted setting stays set
    assert r["ms"] < r["default_ms"]


def test_gain_inside_noise_keeps_defaults():
    # 0.5% better on paper, 5% run-to-run noise: the defaults stay
    eng = FakeEngine(factors={("beta", 48.0): 0.995}, noise=0.05, seed=3)
    start = eng.tunables()
    r = autotune.tune_engine(eng, [1, 2], 0)
    assert r["adopted"] == "defaults" and not r["gain_beyond_noise"]
    assert r["params"] == start
    assert eng.tunables() == start


def test_setting_that_changes_depths_is_refused():
    eng = FakeEngine(factors={("giant_edges", 4096): 0.5}, noise=0.0, bad=("giant_edges", 4096))
    start = eng.tunables()
    with pytest.raises(RuntimeError, match="changed the depths"):
        autotune.tune_engine(eng, [5], 0)
    assert eng.tunables() == start


def test_single_source_search_covers_every_engine_axis():
    eng = FakeEngine()
    seen = set()
    orig = eng.tune

    def spy(**kw):
        seen.update(k for k, v in kw.items() if v != eng.p.get(k))
        orig(**kw)

    eng.tune = spy
    autotune.tune_engine(eng, [1], 0)
    for name in ("pull_records", "pull_rows", "push_sparse_ratio", "pull_runs", "pull_warp", "push_defer_edges",
                 "ctas_per_sm", "giant_edges", "pull_gather_ratio", "alpha", "beta"):
        assert name in seen, name


def test_multi_source_search_uses_its_own_axes():
    eng = FakeEngine(factors={("ms_compact_l2_div", 6): 0.7}, noise=0.001)
    r = autotune.tune_engine(eng, list(range(64)), 0, multi=True)
    assert r["adopted"] == "tuned" and r["params"]["ms_compact_l2_div"] == 6
    assert r["params"]["pull_warp"] == eng.p["pull_warp"]  # single-source axes untouched


class FakeGraph:
    def __init__(self, E):
        self.E = E


class FakeBatch:
    """A mixed batch whose launch time depends on its parameters."""

    def __init__(self, best=(512, 2, 20.0, 24.0)):
        self.sizes = [1000, 2000]
        self.graphs = [FakeGraph(10_000), FakeGraph(30_000)]
        self.params = {"block_size": 256, "ctas_per_sm": 4, "alpha": 14.0, "beta": 24.0}
        self.best = best
        self.runs = 0

    def set_params(self, b, c, a, bt):
        self.params = {"block_size": b, "ctas_per_sm": c, "alpha": a, "beta": bt}

    def _ms(self):
        p = self.params
        return 1.0 + sum(x != y for x, y in zip((p["block_size"], p["ctas_per_sm"], p["alpha"], p["beta"]),
                                                 self.best))

    def run_device(self, queries, ptr):
        self.runs += 1
        return _Stats(self._ms())

    def run(self, queries):
        return [np.arange(8, dtype=np.uint32) + np.uint32(g) for g, _ in queries], _Stats(self._ms())


def test_batch_tuner_finds_the_best_shape_and_caches_it(tmp_path):
    cache = str(tmp_path / "tune.json")
    queries = [(0, 1), (1, 5), (1, 7)]
    b = FakeBatch(best=(512, 2, 20.0, 24.0))
    r = autotune.tune_batch(b, queries, 0, cache=cache)
    assert not r["cached"] and r["ms"] < r["default_ms"]
    assert (r["params"]["block_size"], r["params"]["ctas_per_sm"], r["params"]["alpha"]) == (512, 2, 20.0)
    assert b.params == r["params"]
    # a second batch of the same shape takes the cached choice without timing
    b2 = FakeBatch(best=(512, 2, 20.0, 24.0))
    r2 = autotune.tune_batch(b2, queries, 0, cache=cache)
    assert r2["cached"] and b2.runs == 0 and b2.params == r["params"]
