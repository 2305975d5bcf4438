"""The bench's checker and summaries on the CPU: oracle_check passes exact
depth rows and flags a row with one planted error (the mistake is planted
in the rows handed to the checker, which is the oracle's side); the
learned-vs-plain summary computes its PCIe roofline from the config-5 and
link extras, and says so when config 5 did not run."""
import numpy as np

import bench
from oracle import oracle as O


def _graph():
    idx, ngh, srcs = bench.rmat24_for_reference(12, 4)
    return idx, ngh, srcs


def test_oracle_check_accepts_exact_rows():
    idx, ngh, srcs = _graph()
    runs = [(s, O.bfs_omp(idx, ngh, int(s), 0xFFFFFFFF, 0)) for s in srcs]
    r = bench.oracle_check(idx, ngh, runs)
    assert r["bit_exact_vs_oracle"] and r["checked"] == len(srcs) and r["mismatched_sources"] == []


def test_oracle_check_flags_a_planted_error():
    idx, ngh, srcs = _graph()
    runs = [(s, O.bfs_omp(idx, ngh, int(s), 0xFFFFFFFF, 0).copy()) for s in srcs]
    d = runs[2][1]
    v = int(np.flatnonzero(d != 0xFFFFFFFF)[5])
    d[v] += 1  # one depth off by one
    r = bench.oracle_check(idx, ngh, runs)
    assert not r["bit_exact_vs_oracle"] and r["mismatched_sources"] == [int(srcs[2])]


def test_oracle_check_with_no_rows_is_not_exact():
    idx, ngh, _ = _graph()
    assert not bench.oracle_check(idx, ngh, [])["bit_exact_vs_oracle"]


def test_learned_batched_vs_plain_summary():
    cold = {"ms": 400.0, "h2d_bytes": 16_000_000_000, "zero_copy_bytes": 200_000_000, "levels": 10,
            "pcie_alg_bytes_per_level": 1.6e9}
    c5 = {"V": 105, "E": 3700, "sources": 128, "batched_learned": {"cold": cold, "warm": {}},
          "plain": {}, "batched_alpha_beta": {}, "speedup_vs_plain_cold": 97.0, "speedup_vs_plain_warm": 23.0,
          "learned_vs_batched_alpha_beta_cold": 1.05, "learned_vs_batched_alpha_beta_warm": 0.99,
          "cpu_baseline": {"value": 1.9}, "parity": {"bit_exact_vs_oracle": True}}
    s = bench.learned_batched_vs_plain({"config5_ooc_batched": c5, "pcie": {"h2d_gbs_measured": 55.0}})
    roof = s["roofline"]
    assert roof["bound"] == "pcie" and roof["traffic"] == 16_200_000_000
    assert abs(roof["achieved"] - 40.5) < 1e-9 and abs(roof["frac"] - 40.5 / 55.0) < 1e-12
    assert roof["alg_bytes"] == 1.6e10
    assert "unavailable" in bench.learned_batched_vs_plain({})
