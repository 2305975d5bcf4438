"""Seeded synthetic workloads of the five benchmark configurations.

Inputs are generated, never downloaded: RMAT graphs (Chakrabarti et al.),
a directed power-law graph with preferential-attachment destinations, and a
block-local web-crawl-like graph.  Seeds are 0x5CA90000 + configuration
index, so every run of a configuration sees the same graph and sources.
"""
from __future__ import annotations

import numpy as np

from . import Csr, PagedGraph

SEED_BASE = 0x5CA90000
PAGESIZE_WORDS = 10 * 1024 * 1024  # FLAGS_pagesize = 10 Mi words (src/app.cuh:38,149)
RMAT_ABC = (0.57, 0.19, 0.19)


def rmat(scale: int, edgefactor: float, config_index: int) -> Csr:
    a, b, c = RMAT_ABC
    return Csr.rmat(scale, edgefactor, a, b, c, seed=SEED_BASE + config_index, scramble=True)


def random_sources(csr: Csr, n: int, seed: int) -> list[int]:
    """n distinct seeded random sources with nonzero out-degree."""
    cand = np.flatnonzero(csr.degree() > 0)
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]


def config1():
    """RMAT scale 16, ef 16; source = max-degree vertex."""
    csr = rmat(16, 16, 0)
    return csr, [int(np.argmax(csr.degree()))]


def config2(scale: int = 24, nsrc: int = 64):
    """RMAT scale 24, ef 16; 64 seeded random sources with nonzero degree."""
    csr = rmat(scale, 16, 1)
    return csr, random_sources(csr, nsrc, SEED_BASE + 1)


def config3(V: int = 41_600_000, E: int = 1_470_000_000, max_degree: int = 1 << 20):
    """Directed power-law graph: out-degree Zipf s=1.9 (capped so that every
    adjacency list fits a 10 Mi-word page), destinations by preferential
    attachment; returns (out-edge CSR, in-edge CSR)."""
    csr = Csr.powerlaw(V, E, 1.9, max_degree, seed=SEED_BASE + 2)
    return csr, csr.transpose()


def config4a(scale: int = 25):
    """RMAT scale 25, ef 16, 64 sources per launch."""
    csr = rmat(scale, 16, 3)
    return csr, random_sources(csr, 64, SEED_BASE + 3)


def config4b(ngraphs: int = 32, nqueries: int = 256, scales=(14, 22), edgefactors=(8, 32)):
    """Mixed batch: ngraphs RMAT graphs with scale and edge factor drawn by
    seed from the given ranges (inclusive), nqueries single-source queries
    (graph uniform at random, source a random vertex with nonzero degree).
    Returns (graphs, [(graph, source), ...], [(scale, edgefactor), ...])."""
    rng = np.random.default_rng(SEED_BASE + 3 + 1000)
    shapes = [(int(rng.integers(scales[0], scales[1] + 1)), int(rng.integers(edgefactors[0], edgefactors[1] + 1)))
              for _ in range(ngraphs)]
    a, b, c = RMAT_ABC
    graphs = [Csr.rmat(s, ef, a, b, c, seed=SEED_BASE + 3 + 2000 + i, scramble=True)
              for i, (s, ef) in enumerate(shapes)]
    cands = [np.flatnonzero(g.degree() > 0) for g in graphs]
    queries = []
    for _ in range(nqueries):
        gi = int(rng.integers(0, ngraphs))
        queries.append((gi, int(rng.choice(cands[gi]))))
    return graphs, queries, shapes


def config5(V: int = 105_000_000, E: int = 3_700_000_000, max_degree: int = 4096):
    """Directed web-crawl-like graph: out-degree power law s=2.1, 90 % of the
    edges inside the source's block of 4096 consecutive ids (distinct ids),
    the rest uniform; returns (out-edge CSR, in-edge CSR).  Out-degrees are
    capped at the block size so that a vertex's local edges fit its block
    (with a higher cap the hubs' surplus would have to leave the block and the
    local share would fall below 90 %)."""
    csr = Csr.web(V, E, 2.1, max_degree, 4096, 0.9, seed=SEED_BASE + 4)
    return csr, csr.transpose()


def paged(csr: Csr, pagesize_words: int = PAGESIZE_WORDS) -> PagedGraph:
    return PagedGraph.from_csr(csr, pagesize_words)
