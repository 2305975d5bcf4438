"""Small, self-contained runs of each kernel family, for profilers.

    python -m scaph_b200.kernel_cases <case> [--scale S] [--reps N]

Each case builds a seeded graph, runs the kernels of one family a few times
and exits 0; a profiler pointed at the process (one kernel name, a few
launches) then sees that family on a realistic input larger than L2.

cases:
  bfs      single-source BFS, host-driven level loop (k_push, k_push_giant,
           k_pull as separate launches), RMAT-S, alpha/beta
  graph    the same traversals as one CUDA-graph launch each
  msbfs    64-source multi-source BFS (k_ms_*), RMAT-S
  web      128-source multi-source BFS on the web-like graph of the
           out-of-core batched configuration at 1/2^(25-S) of its size
           (S=25: 105 M vertices), resident, with its transposed pages
  batch    mixed batch of 64 queries over 8 RMAT graphs (k_bt_*), one launch
  pager    out-of-core BFS through a small page pool (k_page_counts, copies,
           zero-copy reads), RMAT-S
  mlp      scheduler network: training steps, forward calls and the
           device timing of both (k_gemm, k_bce, k_adam, k_forward1)
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import DIR_ALPHABETA, Batch, Csr, Engine, Mlp, PagedGraph

SEED = 0x5CA90000


def _rmat(scale: int, seed: int = SEED + 1) -> Csr:
    return Csr.rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed, scramble=True)


def _sources(csr: Csr, n: int, seed: int) -> list[int]:
    cand = np.flatnonzero(csr.degree() > 0)
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]


def case_bfs(scale: int, reps: int, graph_mode: bool) -> str:
    csr = _rmat(scale)
    g = PagedGraph.from_csr(csr)
    eng = Engine(g, direction=DIR_ALPHABETA, use_graph=0 if graph_mode else 2)
    ms = 0.0
    for s in _sources(csr, reps, SEED + 1):
        _, _, st = eng.bfs(s)
        ms += st.ms
    eng.close()
    return f"{reps} BFS on RMAT-{scale} (V={csr.V}, E={csr.E}): {ms / reps:.3f} ms each"


def case_msbfs(scale: int, reps: int) -> str:
    csr = _rmat(scale)
    g = PagedGraph.from_csr(csr)
    eng = Engine(g)
    srcs = _sources(csr, 64, SEED + 3)
    ms = 0.0
    for _ in range(reps):
        _, st = eng.msbfs(srcs)
        ms += st.ms
    eng.close()
    return f"{reps} x 64-source MS-BFS on RMAT-{scale}: {ms / reps:.3f} ms each"


def case_web(scale: int, reps: int) -> str:
    from . import workloads
    f = 2.0 ** (scale - 25)
    csr, tcsr = workloads.config5(V=int(105_000_000 * f), E=int(3_700_000_000 * f))
    g, gt = PagedGraph.from_csr(csr), PagedGraph.from_csr(tcsr)
    eng = Engine(g, gt)
    srcs = _sources(csr, 128, SEED + 4)
    ms = 0.0
    for _ in range(reps):
        _, st = eng.msbfs(srcs)
        ms += st.ms
    eng.close()
    return f"{reps} x 128-source MS-BFS on the web-like graph (V={csr.V}, E={csr.E}): {ms / reps:.3f} ms each"


def case_batch(scale: int, reps: int) -> str:
    graphs = [_rmat(max(10, scale - 4 + (i % 4)), seed=SEED + 3000 + i) for i in range(8)]
    rng = np.random.default_rng(SEED + 3)
    queries = []
    for _ in range(64):
        gi = int(rng.integers(0, len(graphs)))
        queries.append((gi, int(rng.choice(np.flatnonzero(graphs[gi].degree() > 0)))))
    b = Batch(graphs)
    ms = 0.0
    for _ in range(reps):
        _, st = b.run(queries)
        ms += st.ms
    b.close()
    return f"{reps} mixed batches (64 queries, 8 graphs): {ms / reps:.3f} ms each"


def case_pager(scale: int, reps: int) -> str:
    csr = _rmat(scale)
    g = PagedGraph.from_csr(csr, pagesize_words=1 << 18)
    eng = Engine(g, pool_bytes=max(1, g.npages // 4) * g.pagesize * 4)
    ms = 0.0
    for i, s in enumerate(_sources(csr, reps, SEED + 5)):
        eng.evict_all()
        _, _, st = eng.bfs(s)
        ms += st.ms
    eng.close()
    return f"{reps} cold out-of-core BFS on RMAT-{scale} ({g.npages} pages, pool of {max(1, g.npages // 4)}): " \
           f"{ms / reps:.3f} ms each"


def case_mlp(scale: int, reps: int) -> str:
    npages = 64
    net = Mlp(16 + npages, 1 + npages, seed=3)
    rng = np.random.default_rng(7)
    X = rng.random((256, 16 + npages), dtype=np.float32)
    T = (rng.random((256, 1 + npages)) > 0.5).astype(np.float32)
    W = np.full_like(T, 1.0 / T.size)
    t0 = time.perf_counter()
    net.train(X, T, W, epochs=reps, batch=256, lr=1e-3)
    for _ in range(reps):
        net.forward(X[:1])
    dev = net.time(n=256, reps=reps)  # CUDA-event timing; launches the single-row kernel k_forward1
    return (f"{reps} training steps and {reps} single-row forward calls: {time.perf_counter() - t0:.3f} s; "
            f"device us: {dev}")


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("case", choices=["bfs", "graph", "msbfs", "web", "batch", "pager", "mlp"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--reps", type=int, default=4)
    a = ap.parse_args(argv)
    if a.case in ("bfs", "graph"):
        msg = case_bfs(a.scale, a.reps, a.case == "graph")
    elif a.case == "msbfs":
        msg = case_msbfs(a.scale, a.reps)
    elif a.case == "web":
        msg = case_web(a.scale, a.reps)
    elif a.case == "batch":
        msg = case_batch(a.scale, a.reps)
    elif a.case == "pager":
        msg = case_pager(a.scale, a.reps)
    else:
        msg = case_mlp(a.scale, a.reps)
    print(msg, flush=True)


if __name__ == "__main__":
    main()
