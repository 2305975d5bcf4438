"""Small seeded graphs shared by the tests (built with the library's generators
or directly as numpy CSR arrays)."""
from __future__ import annotations

import numpy as np

import scaph_b200 as S

SEED = 0x5CA90000


def csr_from_edges(V: int, src, dst, symmetric: bool = False) -> S.Csr:
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    if symmetric:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    keep = src != dst
    src, dst = src[keep], dst[keep]
    key = np.unique(src * V + dst)
    s, d = key // V, key % V
    idx = np.zeros(V + 1, np.uint64)
    np.add.at(idx, s + 1, 1)
    idx = np.cumsum(idx, dtype=np.uint64)
    return S.Csr.from_arrays(idx, d.astype(np.uint32))


def path(V: int) -> S.Csr:
    a = np.arange(V - 1)
    return csr_from_edges(V, a, a + 1, symmetric=True)


def star(V: int, center: int = 0) -> S.Csr:
    leaves = np.array([v for v in range(V) if v != center])
    return csr_from_edges(V, np.full(len(leaves), center), leaves, symmetric=True)


def random_graph(V: int, E: int, seed: int, symmetric: bool = True) -> S.Csr:
    rng = np.random.default_rng(seed)
    return csr_from_edges(V, rng.integers(0, V, E), rng.integers(0, V, E), symmetric=symmetric)


def sources(csr: S.Csr, n: int, seed: int) -> list[int]:
    """n seeded random sources with nonzero out-degree (plus none if none exist)."""
    deg = csr.degree()
    cand = np.flatnonzero(deg > 0)
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]
