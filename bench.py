#!/usr/bin/env python3
"""BFS benchmark of the sm_100a Scaph engine.

Workload (default): RMAT scale 24, edge factor 16, a/b/c/d = .57/.19/.19/.05,
seeded, symmetrised, deduplicated, uint32 ids, paged CSR with 10 Mi-word
pages, fully resident in HBM; 64 seeded random sources with nonzero degree,
each run separately; Beamer alpha/beta direction switch (alpha 14, beta 96).
One step = one single-source BFS.  GTEPS follows the reference's formula,
edge_count / traversal time (src/app.cuh:252).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are replicas: each rank runs its own BFS sources on its own
copy of the graph (no collective on the data path); value = all ranks'
traversed edges / max-over-ranks time.

--impl reference times the reference's own CPU BFS (bfs::check,
app/bfs.cu:67-117, compiled from the reference sources into oracle/_ref) on
the host cores, one process per core, on the same graph and sources.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BFS GTEPS (edge_count / traversal time), plain direction-optimizing engine, RMAT-24 in HBM"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
NOMINAL_HBM_GBS = 8000.0


# Measured DRAM bytes (read + write) per k_pull launch on RMAT-24: ncu's dram__bytes_read.sum
# + dram__bytes_write.sum (a 1-pass metric set) over 5 k_pull launches (-s 3 -c 5) of
# `bench.py --host-loop --steps 2 --warmup 1 --no-cpu --no-extras --no-tune`, mean per launch.
K_PULL_TRAFFIC_BYTES = 133_429_000


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2048)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations (rank 0, N=1 only anyway)")
    ap.add_argument("--no-config5", action="store_true",
                    help="skip the 105M-vertex / 3.7B-edge web graph (about a minute to generate)")
    ap.add_argument("--only-extra", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner report")
    ap.add_argument("--host-loop", action="store_true",
                    help="time the host-driven level loop (one launch per level kernel) instead of one "
                         "CUDA-graph launch per BFS; for profilers that time kernels one launch at a time")
    return ap.parse_args()


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.out.flush()
        self.out.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.out.name)
        load = [x for x in sm if smax and x > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def config_dict(V, E, scale, nsrc):
    """The workload's description; identical in both arms."""
    return {"workload": f"rmat{scale}-ef16 single-source BFS, {nsrc} seeded sources, alpha/beta 14/96, in HBM",
            "graph": f"RMAT scale {scale}, ef 16, a/b/c/d .57/.19/.19/.05, symmetrised, dedup",
            "V": V, "E": E, "sources": nsrc, "pagesize_words": 10 * 1024 * 1024,
            "l2": "inputs larger than L2 (paged graph %.2f GB > 126 MB)" % (4 * (3 * V + E) / 1e9)}


# ---------------------------------------------------------------------------
# the checker: depths against the CPU oracle (outside every timed region)
# ---------------------------------------------------------------------------
def oracle_check(idx, ngh, runs, unreached=0xFFFFFFFF, threads=0):
    """runs: (source, uint32 depth array) pairs.  Each is compared bit for bit
    with the level-synchronous restatement of bfs::check (app/bfs.cu:70-101)
    run with OpenMP on the host cores."""
    import numpy as np

    from oracle import oracle as O

    n, bad, t0 = 0, [], time.perf_counter()
    for src, depth in runs:
        ref = O.bfs_omp(idx, ngh, int(src), unreached, threads)
        n += 1
        if not np.array_equal(np.asarray(depth).view(np.uint32), ref):
            bad.append(int(src))
    return {"bit_exact_vs_oracle": n > 0 and not bad, "checked": n, "mismatched_sources": bad[:8],
            "oracle": "level-synchronous bfs::check restatement, OpenMP", "check_s": round(time.perf_counter() - t0, 1)}


# ---------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------
_W = {}


def _ref_worker_init(idx_path, ngh_path):
    import numpy as np

    from oracle import oracle as O

    _W["idx"] = np.load(idx_path, mmap_mode="r")
    _W["ngh"] = np.load(ngh_path, mmap_mode="r")
    _W["O"] = O
    _W["vals"] = np.zeros(len(_W["idx"]) - 1, np.uint32)


def _ref_worker_bfs(src):
    O = _W["O"]
    if O.ref_available():
        _, sec = O.ref_bfs_check(_W["idx"], _W["ngh"], src, _W["vals"])
        return sec
    t = time.perf_counter()
    O.bfs(_W["idx"].astype("uint64"), _W["ngh"], src, 63)
    return time.perf_counter() - t


def rmat24_for_reference(scale, nsrc):
    """The headline graph and sources, built without the product library:
    the oracle's RMAT generator (identical CSR to scaph_gen_rmat, checked by
    a CPU test) and the same seeded choice of sources as
    scaph_b200.workloads.config2."""
    import numpy as np

    from oracle import oracle as O

    seed = 0x5CA90000 + 1
    idx, ngh = O.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed, True)
    cand = np.flatnonzero(np.diff(idx) > 0)
    rng = np.random.default_rng(seed)
    srcs = [int(x) for x in rng.choice(cand, size=min(nsrc, len(cand)), replace=False)]
    return idx, ngh, srcs


def run_reference(args, world):
    import multiprocessing as mp

    import numpy as np

    from oracle import oracle as O

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    idx, ngh, srcs = rmat24_for_reference(args.scale, args.sources)
    V, E = len(idx) - 1, len(ngh)
    kind = "reference" if O.ref_available() else "port"
    tmp = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    idx_path, ngh_path = os.path.join(tmp, "idx.npy"), os.path.join(tmp, "ngh.npy")
    np.save(idx_path, idx.astype(np.uint32))
    np.save(ngh_path, ngh)
    del idx, ngh
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_worker_init, initargs=(idx_path, ngh_path)) as pool:
        pool.map(_ref_worker_bfs, [srcs[i % len(srcs)] for i in range(max(args.warmup, cores))])
        order = [srcs[i % len(srcs)] for i in range(args.steps)]
        t0 = time.perf_counter()
        secs = pool.map(_ref_worker_bfs, order, chunksize=1)
        wall = time.perf_counter() - t0
    for p in (idx_path, ngh_path):
        os.unlink(p)
    os.rmdir(tmp)
    value = args.steps * E / wall / 1e9
    sample = (f"{args.steps} single-source BFS of bfs::check over the flat CSR, {cores} processes "
              f"(one source each), mean {statistics.mean(secs):.3f} s per source")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded RMAT)", "config": config_dict(V, E, args.scale, len(srcs)),
            "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# CPU baseline beside our own arm (rank 0, N = 1)
# ---------------------------------------------------------------------------
def cpu_baseline(csr, srcs, budget_s):
    import numpy as np

    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    idx32 = csr.idx.astype(np.uint32) if kind == "reference" else None
    vals = np.zeros(csr.V, np.uint32)
    n, tot = 0, 0.0
    for s in srcs:
        if kind == "reference":
            _, sec = O.ref_bfs_check(idx32, csr.ngh, s, vals)
        else:
            t = time.perf_counter()
            O.bfs(csr.idx, csr.ngh, s, 63)
            sec = time.perf_counter() - t
        n += 1
        tot += sec
        if tot >= budget_s:
            break
    out = {"value": n * csr.E / tot / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind,
           "sample": f"{n} of the {len(srcs)} sources, single-threaded bfs::check "
                     f"({'reference code' if kind == 'reference' else 'oracle restatement'}), "
                     f"{tot:.1f} s total"}
    # beside it, the level-synchronous restatement with OpenMP on every host core
    # (same depths by construction), on the same sources for up to a third of the budget
    cores = os.cpu_count() or 1
    m, t_omp = 0, 0.0
    for s in srcs:
        t = time.perf_counter()
        O.bfs_omp(csr.idx, csr.ngh, s, 63, cores)
        t_omp += time.perf_counter() - t
        m += 1
        if t_omp >= budget_s / 3:
            break
    out["openmp"] = {"value": m * csr.E / t_omp / 1e9, "unit": "GTEPS", "cores": cores, "kind": "port",
                     "sample": f"{m} of the {len(srcs)} sources, level-synchronous restatement, "
                               f"OpenMP on {cores} threads, {t_omp:.1f} s total"}
    return out


# ---------------------------------------------------------------------------
# the other configurations (reported beside the headline, rank 0, N = 1)
# ---------------------------------------------------------------------------
def extra_config1():
    """RMAT-16, max-degree source, checked bit-exact against the oracle."""
    import numpy as np

    import scaph_b200 as S
    from oracle import oracle as O
    from scaph_b200 import workloads

    csr, (src,) = workloads.config1()
    g = workloads.paged(csr)
    eng = S.Engine(g)
    eng.bfs(src)
    d, _, st = eng.bfs(src)
    ok = bool(np.array_equal(d, O.bfs(csr.idx, csr.ngh, src)))
    eng.close()
    return {"graph": "RMAT-16 ef16", "V": csr.V, "E": csr.E, "source": src, "levels": st.levels,
            "ms": st.ms, "gteps": csr.E / (st.ms / 1e3) / 1e9, "bit_exact_vs_oracle": ok}


def extra_config4a(stream):
    """RMAT-25: 64 sources in one multi-source launch vs 64 plain runs."""
    import torch

    import scaph_b200 as S
    from scaph_b200 import workloads

    csr, srcs = workloads.config4a()
    g = workloads.paged(csr)
    eng = S.Engine(g, stream=stream.cuda_stream)
    out = torch.empty((len(srcs), csr.V), dtype=torch.int32, device="cuda")
    from scaph_b200 import autotune

    tune = autotune.tune_engine(eng, workloads.random_sources(csr, 64, workloads.SEED_BASE + 203), out.data_ptr(),
                                multi=True, repeats=2)
    eng.msbfs_device(srcs, out.data_ptr())
    runs = [eng.msbfs_device(srcs, out.data_ptr()) for _ in range(3)]
    ms_batch = min(r.ms for r in runs)
    tr = eng.msbfs_trace()
    eng.tune(alpha=14.0, beta=24.0)  # the plain engine keeps the default alpha/beta
    d = torch.empty(csr.V, dtype=torch.int32, device="cuda")
    for s in srcs[:3]:
        eng.bfs_device(s, d.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in srcs:
        eng.bfs_async(s, d.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1)
    eng.close()
    n = len(srcs)
    # every row of the batched launch against the CPU oracle (untimed)
    parity = oracle_check(csr.idx, csr.ngh, ((s, out[i].cpu().numpy()) for i, s in enumerate(srcs)))
    return {"graph": "RMAT-25 ef16", "V": csr.V, "E": csr.E, "sources_per_launch": n, "parity": parity,
            "autotune": tune,
            "batched_ms": ms_batch, "batched_gteps_per_source": n * csr.E / (ms_batch / 1e3) / 1e9,
            "plain_ms_for_same_sources": ms_plain, "plain_gteps": n * csr.E / (ms_plain / 1e3) / 1e9,
            "speedup_vs_plain": ms_plain / ms_batch, "levels": len(tr),
            "directions": "".join("p" if t["direction"] else "P" for t in tr)}


def extra_config4b(stream):
    """Mixed batch: 256 single-source queries over 32 RMAT graphs (scales
    14-22, edge factors 8-32, drawn by seed) in one CUDA-graph launch with
    autotuned parameters, against the plain engine running the same queries
    one by one (one engine per graph, one graph launch per query)."""
    import numpy as np
    import torch

    import scaph_b200 as S
    from scaph_b200 import autotune, workloads

    t0 = time.time()
    graphs, queries, shapes = workloads.config4b()
    gen_s = time.time() - t0
    b = S.Batch(graphs, stream=stream.cuda_stream)
    words = b.out_words(queries)
    out = torch.empty(words, dtype=torch.int32, device="cuda")
    with tempfile.TemporaryDirectory() as td:
        tune = autotune.tune_batch(b, queries, out.data_ptr(), repeats=2, cache=os.path.join(td, "tune.json"))
    runs = [b.run_device(queries, out.data_ptr()) for _ in range(5)]
    ms_batch = min(r.ms for r in runs)
    tr = b.trace()
    # plain: one engine per graph, every query its own graph launch
    engines = [S.Engine(S.PagedGraph.from_csr(g), stream=stream.cuda_stream) for g in graphs]
    ref = torch.empty(words, dtype=torch.int32, device="cuda")
    offs, o = [], 0
    for gi, _ in queries:
        offs.append(o)
        o += graphs[gi].V
    for (gi, s), off in zip(queries[:8], offs):
        engines[gi].bfs_device(s, ref.data_ptr() + 4 * off)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for (gi, s), off in zip(queries, offs):
        engines[gi].bfs_async(s, ref.data_ptr() + 4 * off)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1)
    exact = bool(torch.equal(out, ref))
    # every query's row against the CPU oracle on its own graph (untimed)
    host = out.cpu().numpy()
    parity = {"checked": 0, "mismatched_sources": [], "check_s": 0.0}
    for (gi, src), off in zip(queries, offs):
        r = oracle_check(graphs[gi].idx, graphs[gi].ngh, [(src, host[off:off + graphs[gi].V])])
        parity["checked"] += r["checked"]
        parity["check_s"] += r["check_s"]
        if r["mismatched_sources"]:
            parity["mismatched_sources"].append([gi, src])
    parity["bit_exact_vs_oracle"] = parity["checked"] == len(queries) and not parity["mismatched_sources"]
    for e in engines:
        e.close()
    b.close()
    teps = sum(graphs[gi].E for gi, _ in queries)
    per_graph = np.bincount([gi for gi, _ in queries], minlength=len(graphs))
    return {"graphs": len(graphs), "queries": len(queries), "V_total": sum(g.V for g in graphs),
            "E_total": sum(g.E for g in graphs), "scales": [sc for sc, _ in shapes],
            "edgefactors": [ef for _, ef in shapes], "max_queries_per_graph": int(per_graph.max()),
            "graph_gen_s": round(gen_s, 1), "launches_per_batch": runs[-1].launches,
            "batched_ms": ms_batch, "batched_gteps": teps / (ms_batch / 1e3) / 1e9,
            "plain_ms": ms_plain, "plain_gteps": teps / (ms_plain / 1e3) / 1e9,
            "speedup_vs_plain": ms_plain / ms_batch, "bit_exact_vs_plain": exact, "parity": parity,
            "levels": len(tr),
            "directions": "".join("p" if t["direction"] else "P" for t in tr),
            "autotune": {"params": tune["params"], "default_ms": tune["default_ms"], "tuned_ms": tune["ms"],
                         "candidates": tune["tried"], "seconds": round(tune["seconds"], 1)}}


def _digest(a):
    import hashlib

    import numpy as np

    return hashlib.blake2b(memoryview(np.ascontiguousarray(a)), digest_size=16).hexdigest()


def _run_set(S, g, gt, srcs, pool, net=None, cold=False, warm_pass=True, digests=None, **kw):
    """Times `srcs`; returns total ms, PCIe bytes, levels.  With `digests`
    (source -> list), a digest of every checked source's depths is added."""
    eng = S.Engine(g, gt, pool_bytes=pool, direction=S.DIR_LEARNED if net else 0, **kw)
    if net:
        eng.set_scheduler(net)
    if warm_pass and not cold:
        for s in srcs:
            eng.bfs(s)
    ms, h2d, zc, alg, levels, level_ms = 0.0, 0, 0, 0, 0, 0.0
    for s in srcs:
        if cold:
            eng.evict_all()
        d, _, st = eng.bfs(s)
        ms += st.ms
        h2d += st.h2d_bytes
        zc += st.zc_bytes
        alg += st.pcie_alg_bytes
        levels += st.levels
        level_ms += sum(t["ms"] for t in eng.trace())
        if digests is not None and s in digests:
            digests[s].append(_digest(d))
    eng.close()
    return {"ms": ms, "h2d_bytes": h2d, "zc_bytes": zc, "pcie_alg_bytes": alg, "levels": levels, "level_ms": level_ms}


def extra_config2_learned(stream, nsrc_train=16):
    """The headline graph (RMAT-24 in HBM) with the learned direction: the
    network trained on dual-timed plain runs of 16 other sources, evaluated
    on the 64 headline sources as one CUDA-graph launch each (the decision
    runs on the device, k_decide_learned), against the plain alpha/beta
    engine on the same sources; depths compared with the plain engine's."""
    import torch

    import scaph_b200 as S
    from scaph_b200 import scheduler, workloads

    csr, srcs = workloads.config2()
    g = workloads.paged(csr)
    train = [s for s in workloads.random_sources(csr, nsrc_train + len(srcs), workloads.SEED_BASE + 205)
             if s not in set(srcs)][:nsrc_train]
    traces = scheduler.collect(g, None, train)
    net, info = scheduler.train(traces, g, None, g.npages, 0.0, epochs=200)
    d0 = torch.empty(csr.V, dtype=torch.int32, device="cuda")
    d1 = torch.empty(csr.V, dtype=torch.int32, device="cuda")
    plain = S.Engine(g, stream=stream.cuda_stream)
    learned = S.Engine(g, stream=stream.cuda_stream, direction=S.DIR_LEARNED)
    learned.set_scheduler(net)
    exact = True
    for s in srcs:
        plain.bfs_device(s, d0.data_ptr())
        learned.bfs_device(s, d1.data_ptr())
        exact &= bool(torch.equal(d0, d1))
    out = {"graph": "RMAT-24 ef16 (the headline graph)", "train_sources": len(train), "eval_sources": len(srcs),
           "training": info, "depths_equal_plain": exact}
    for name, eng, d in (("plain", plain, d0), ("learned", learned, d1)):
        for s in srcs[:3]:
            eng.bfs_async(s, d.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(4):
            for s in srcs:
                eng.bfs_async(s, d.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / (4 * len(srcs))
        out[name] = {"ms_per_bfs": ms, "gteps": csr.E / (ms / 1e3) / 1e9}
        eng.close()
    out["speedup"] = out["plain"]["ms_per_bfs"] / out["learned"]["ms_per_bfs"]
    return out


def extra_config3(nsrc_train=32, nsrc_eval=32, nsrc_oracle=16):
    """Directed power law 41.6M / 1.47B: the learned scheduler (trained on
    dual-timed plain runs of 32 sources) against alpha/beta + demand paging
    on 32 held-out sources, in HBM and out of core with the 12 GB page pool
    (warm: steady-state serving; cold: every source starts from an empty
    pool).  The depths of the first 16 held-out sources, in every regime and
    both arms, are checked against the CPU oracle (digests)."""
    import time as _t

    import scaph_b200 as S
    from scaph_b200 import scheduler, workloads

    t0 = _t.time()
    csr, tcsr = workloads.config3()
    g, gt = workloads.paged(csr), workloads.paged(tcsr)
    del tcsr
    gen_s = _t.time() - t0
    srcs = workloads.random_sources(csr, nsrc_train + nsrc_eval, workloads.SEED_BASE + 2)
    train, held = srcs[:nsrc_train], srcs[nsrc_train:]
    pool = 12 * 10**9
    nslots = pool // (g.pagesize * 4)
    page_ms = g.pagesize * 4 / 50e9 * 1e3  # page copy at ~50 GB/s (PCIe Gen5 x16, pinned)
    traces = scheduler.collect(g, gt, train)
    net, info = scheduler.train(traces, g, gt, nslots, page_ms, epochs=200)
    info["held_out"] = scheduler.held_out_accuracy(net, scheduler.collect(g, gt, held), g, gt, nslots, page_ms)
    E, n = csr.E, len(held)
    res = {"graph": "directed power law, Zipf 1.9 out-degree, preferential-attachment destinations",
           "V": csr.V, "E": E, "out_pages": g.npages, "in_pages": gt.npages, "pool_bytes": pool,
           "graph_gen_s": round(gen_s, 1), "train_sources": nsrc_train, "eval_sources": n, "training": info}
    digests = {s: [] for s in held[:nsrc_oracle]}
    for name, kw in (("hbm", dict(pool=0, use_graph=0)), ("ooc_warm", dict(pool=pool)),
                     ("ooc_cold", dict(pool=pool, cold=True))):
        plain = _run_set(S, g, gt, held, kw["pool"], None, cold=kw.get("cold", False),
                         use_graph=kw.get("use_graph", 0), digests=digests)
        learned = _run_set(S, g, gt, held, kw["pool"], net, cold=kw.get("cold", False),
                           use_graph=kw.get("use_graph", 0) if kw["pool"] else 0, digests=digests)
        res[name] = {
            "plain_gteps": n * E / (plain["ms"] / 1e3) / 1e9, "learned_gteps": n * E / (learned["ms"] / 1e3) / 1e9,
            "speedup": plain["ms"] / learned["ms"],
            "plain_pcie_bytes_per_level": plain["h2d_bytes"] / max(1, plain["levels"]),
            "learned_pcie_bytes_per_level": learned["h2d_bytes"] / max(1, learned["levels"]),
            "plain_zero_copy_bytes": plain["zc_bytes"], "learned_zero_copy_bytes": learned["zc_bytes"],
            # the least the levels had to move over the link (non-resident
            # active words, get_page_info's datas) against what moved
            "plain_pcie_alg_bytes_per_level": plain["pcie_alg_bytes"] / max(1, plain["levels"]),
            "learned_pcie_alg_bytes_per_level": learned["pcie_alg_bytes"] / max(1, learned["levels"]),
            "plain_ms": plain["ms"], "learned_ms": learned["ms"],
            # device time inside the levels (the rest of ms is the host loop
            # between them: page decisions, features, the network)
            "plain_level_ms": plain["level_ms"], "learned_level_ms": learned["level_ms"],
            "plain_moved_bytes": plain["h2d_bytes"] + plain["zc_bytes"],
            "learned_moved_bytes": learned["h2d_bytes"] + learned["zc_bytes"]}
    # the checker: oracle depths of the checked held-out sources against the
    # six runs of each (plain and learned, three regimes)
    from oracle import oracle as O

    t1, bad = _t.perf_counter(), []
    for s, ds in digests.items():
        ref = _digest(O.bfs_omp(csr.idx, csr.ngh, s))
        if len(ds) != 6 or any(d != ref for d in ds):
            bad.append(s)
    res["parity"] = {"bit_exact_vs_oracle": not bad, "checked": len(digests), "runs_per_source": 6,
                     "mismatched_sources": bad[:8], "check_s": round(_t.perf_counter() - t1, 1),
                     "oracle": "level-synchronous bfs::check restatement, OpenMP (depth digests)"}
    return res


def extra_config5(stream, nsrc=128, nplain=8, ntrain=8):
    """Web-crawl-like graph 105M / 3.7B streamed out of core with a 24 GB page
    pool: 128 sources per multi-source launch - with alpha/beta, with the
    scheduler's page-traffic rule alone, and with the learned scheduler
    (network trained on this graph's plain-engine traces and on two
    multi-source batches of other sources; direction stays alpha/beta, and
    the push levels the network or the frontier's growth mark as leading
    into the pull levels prefetch the in-pages the first pull level reads) -
    against the plain engine (one source per launch, alpha/beta + demand
    paging), warm and cold pools."""
    import torch

    import numpy as np

    import scaph_b200 as S
    from scaph_b200 import scheduler, workloads

    t0 = time.time()
    csr, csr_t = workloads.config5()
    g, gt = workloads.paged(csr), workloads.paged(csr_t)
    srcs = workloads.random_sources(csr, nsrc, workloads.SEED_BASE + 4)
    pool_train = [s for s in workloads.random_sources(csr, 2 * nsrc + ntrain + nsrc, workloads.SEED_BASE + 104)
                  if s not in set(srcs)]
    gen_s = time.time() - t0
    V, E = csr.V, csr.E
    del csr_t  # the paged copies are what the engines use (csr stays for the checker)
    pool = 24_000_000_000
    nslots = pool // (g.pagesize * 4)
    out = {"graph": "web-like: power-law out-degree s=2.1, 90% of edges inside 4096-id blocks", "V": V, "E": E,
           "out_pages": g.npages, "in_pages": gt.npages, "pool_bytes": pool,
           "pool_pages": nslots, "graph_gen_s": round(gen_s, 1), "sources": nsrc}
    depth = torch.empty((nsrc, V), dtype=torch.int32, device="cuda")
    # the scheduler network, trained on this graph (sources disjoint from the
    # evaluated ones)
    t1 = time.time()
    page_ms = g.pagesize * 4 / 50e9 * 1e3
    traces = scheduler.collect(g, gt, pool_train[:ntrain])
    ms_rows = scheduler.collect_ms(g, gt, [pool_train[ntrain:ntrain + nsrc], pool_train[ntrain + nsrc:ntrain + 2 * nsrc]],
                                   depth_ptr=depth.data_ptr())
    net, info = scheduler.train(traces, g, gt, nslots, page_ms, epochs=200, ms_rows=ms_rows)
    info["collect_and_train_s"] = round(time.time() - t1, 1)
    out["training"] = info
    arms = (("batched_alpha_beta", S.DIR_ALPHABETA, None), ("batched_transfer_rule", S.DIR_LEARNED, None),
            ("batched_learned", S.DIR_LEARNED, net))
    for name, direction, sched in arms:
        eng = S.Engine(g, gt, pool_bytes=pool, direction=direction, stream=stream.cuda_stream)
        if sched is not None:
            eng.set_scheduler(sched)
        res = {}
        for regime in ("cold", "warm"):
            if regime == "cold":
                eng.evict_all()
            st = eng.msbfs_device(srcs, depth.data_ptr())
            tr = eng.msbfs_trace()
            res[regime] = {"ms": st.ms, "gteps_per_source": nsrc * E / (st.ms / 1e3) / 1e9,
                           "h2d_bytes": st.h2d_bytes, "zero_copy_bytes": st.zc_bytes,
                           "page_faults": st.page_faults, "prefetched": st.prefetched, "levels": st.levels,
                           "pcie_bytes_per_level": (st.h2d_bytes + st.zc_bytes) / max(1, st.levels),
                           "pcie_alg_bytes_per_level": st.pcie_alg_bytes / max(1, st.levels),
                           "directions": "".join("p" if t["direction"] else "P" for t in tr),
                           "level_ms": [round(float(t["ms"]), 2) for t in tr],
                           "gap_ms": [round(float(t["push_ms"]), 2) for t in tr],
                           "host_ms": [round(float(t["pull_ms"]), 2) for t in tr],
                           "level_h2d_mb": [round(int(t["h2d_bytes"]) / 1e6, 1) for t in tr]}
        out[name] = res
        eng.close()
    # plain engine, one source per launch, on the first sources
    eng = S.Engine(g, gt, pool_bytes=pool, stream=stream.cuda_stream)
    d1 = torch.empty(V, dtype=torch.int32, device="cuda")
    plain = {}
    for regime in ("cold", "warm"):
        ms, h2d, zc, alg, lv, exact = 0.0, 0, 0, 0, 0, True
        for i, s in enumerate(srcs[:nplain]):
            if regime == "cold":
                eng.evict_all()
            st = eng.bfs_device(s, d1.data_ptr())
            ms += st.ms
            h2d += st.h2d_bytes
            zc += st.zc_bytes
            alg += st.pcie_alg_bytes
            lv += st.levels
            exact &= bool(torch.equal(d1, depth[i]))
        plain[regime] = {"ms_per_source": ms / nplain, "gteps": E / (ms / nplain / 1e3) / 1e9,
                         "pcie_bytes_per_source": (h2d + zc) / nplain, "pcie_bytes_per_level": (h2d + zc) / max(1, lv),
                         "pcie_alg_bytes_per_level": alg / max(1, lv), "batched_rows_equal": exact}
    eng.close()
    out["plain"] = plain
    out["plain_sources_timed"] = nplain
    for regime in ("cold", "warm"):
        out[f"speedup_vs_plain_{regime}"] = out["batched_learned"][regime]["gteps_per_source"] / plain[regime]["gteps"]
        out[f"learned_vs_batched_alpha_beta_{regime}"] = (out["batched_alpha_beta"][regime]["ms"] /
                                                        out["batched_learned"][regime]["ms"])
    # the checker: rows of the last (learned, warm) batched launch against the
    # CPU oracle, untimed; the oracle's own time on those sources is the CPU
    # baseline (level-synchronous bfs::check restatement, OpenMP, every core)
    nchk = max(nplain, 8)
    out["parity"] = oracle_check(csr.idx, csr.ngh, ((s, depth[i].cpu().numpy()) for i, s in enumerate(srcs[:nchk])))
    cpu_s = out["parity"]["check_s"]
    out["cpu_baseline"] = {"value": nchk * E / max(cpu_s, 1e-9) / 1e9, "unit": "GTEPS per source",
                           "cores": os.cpu_count() or 1, "kind": "port",
                           "sample": f"{nchk} sources of the same graph, level-synchronous restatement of bfs::check "
                                     f"with OpenMP, {cpu_s:.1f} s (includes comparing the rows)"}
    return out


def learned_batched_vs_plain(extras):
    """The metric's own comparison, from the config-5 and PCIe extras:
    learned+batched against the plain engine on the largest out-of-core
    configuration, GTEPS per source and PCIe bytes per level (actual and
    algorithmic), with the PCIe roofline of the cold batched launch."""
    c5, pc = extras.get("config5_ooc_batched") or {}, extras.get("pcie") or {}
    if "batched_learned" not in c5:
        return {"unavailable": c5.get("error", "config 5 not run")}
    link = pc.get("h2d_gbs_measured")
    cold = c5["batched_learned"]["cold"]
    moved = cold["h2d_bytes"] + cold["zero_copy_bytes"]
    achieved = moved / (cold["ms"] / 1e3) / 1e9
    return {
        "config": "config 5: web-like graph V=%d E=%d, 24 GB page pool, %d sources per launch" % (
            c5["V"], c5["E"], c5["sources"]),
        "learned_batched": c5["batched_learned"], "plain": c5["plain"],
        "batched_alpha_beta": c5["batched_alpha_beta"],
        "gteps_ratio_cold": c5["speedup_vs_plain_cold"], "gteps_ratio_warm": c5["speedup_vs_plain_warm"],
        "learned_vs_batched_alpha_beta_cold": c5["learned_vs_batched_alpha_beta_cold"],
        "learned_vs_batched_alpha_beta_warm": c5["learned_vs_batched_alpha_beta_warm"],
        "roofline": {"bound": "pcie", "achieved": achieved, "peak": link, "unit": "GB/s",
                     "frac": achieved / link if link else None,
                     "peak_source": "pinned host-to-device copy measured in the same run",
                     "traffic": moved, "alg_bytes": cold["pcie_alg_bytes_per_level"] * cold["levels"]},
        "cpu_baseline": c5["cpu_baseline"], "parity": c5["parity"], "training": c5.get("training")}


def extra_pcie(stream):
    """Pinned host->device copy bandwidth (best of 5, 1 GiB)."""
    import torch

    h = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()
    d = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d.copy_(h, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, (1 << 30) / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del h, d
    return {"h2d_gbs_measured": best, "nominal_gbs": 64.0}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world):
    import numpy as np
    import torch
    import torch.distributed as dist

    import scaph_b200 as S
    from scaph_b200 import replicas, workloads

    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    t0 = time.time()
    csr, srcs = workloads.config2(args.scale, args.sources)
    g = workloads.paged(csr)
    gen_s = time.time() - t0
    V, E = csr.V, csr.E
    # a dedicated (non-default) stream: the engine runs on it and the CUDA
    # events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng = S.Engine(g, device=local_rank, stream=stream.cuda_stream, use_graph=2 if args.host_loop else 0)
    depth = torch.empty(V, dtype=torch.int32, device="cuda")
    # The autotuner on 8 other sources of the same graph, on a separate
    # engine, reported beside the line: the timed engine keeps the library's
    # defaults (A/B runs on whole traversals chose them; a winner on 8
    # tuning sources did not carry over to the timed ones in earlier runs).
    tune = None
    if not args.no_tune:
        from scaph_b200 import autotune

        eng_t = S.Engine(g, device=local_rank, stream=stream.cuda_stream)
        tune = autotune.tune_engine(eng_t, workloads.random_sources(csr, 8, workloads.SEED_BASE + 201),
                                    depth.data_ptr())
        eng_t.close()

    order = replicas.rank_sources(srcs, rank, max(args.steps, args.warmup))

    def src_of(i):
        return order[i % len(order)]

    for i in range(args.warmup):
        eng.bfs_device(src_of(i), depth.data_ptr())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(gpu_index(local_rank))
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(args.steps):  # each BFS is one graph launch; no host sync in between
        eng.bfs_async(src_of(i), depth.data_ptr())
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    # kernels those runs launched (the direction decisions are deterministic,
    # so a counted replay of the same sources launches the same kernels)
    # Every distinct timed source (up to 16 per rank on several GPUs, where
    # the ranks share the host cores) is also checked bit for bit against the
    # CPU oracle, from the same replay.
    launches, g500, parity_runs = 0, [], []
    check_cap = len(srcs) if world == 1 else max(1, 16 // world)
    threads = max(1, (os.cpu_count() or 1) // world)
    seen = set()
    parity = {"checked": 0, "mismatched_sources": [], "check_s": 0.0}
    for i in range(args.steps):
        st = eng.bfs_device(src_of(i), depth.data_ptr())
        launches += st.launches
        g500.append(st.reached_edges / 2 / (st.ms / 1e3) / 1e9)  # Graph500: undirected edges reached
        if src_of(i) not in seen and len(seen) < check_cap:
            seen.add(src_of(i))
            r = oracle_check(csr.idx, csr.ngh, [(src_of(i), depth.cpu().numpy())], threads=threads)
            parity["checked"] += r["checked"]
            parity["mismatched_sources"] += r["mismatched_sources"]
            parity["check_s"] += r["check_s"]
    nbad = len(parity["mismatched_sources"])
    if world > 1:
        t = torch.tensor([parity["checked"], nbad], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        parity["checked"], nbad = int(t[0]), int(t[1])
    parity["bit_exact_vs_oracle"] = parity["checked"] > 0 and nbad == 0
    parity["oracle"] = "level-synchronous bfs::check restatement, OpenMP on %d host threads per rank" % threads
    parity["sources"] = "every distinct timed source" if world == 1 else f"up to {check_cap} timed sources per rank"
    ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    if world > 1:
        dist.barrier()
    value = replicas.aggregate_gteps(world, args.steps, E, ms)

    # end to end through the public API: the source id in, every step's depths
    # copied back into page-locked host memory.  Headline: the pipelined call
    # (scaph_bfs_enqueue: step i's copy overlaps step i+1's traversal, results
    # land in two host buffers used in turn); beside it the synchronous
    # scaph_bfs, one step at a time.
    host_bufs = [S.PinnedArray(V) for _ in range(2)]
    n_e2e = args.steps

    def timed_e2e(step):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev2.record(stream)
        for i in range(n_e2e):
            step(i)
        eng.sync()
        ev3.record(stream)
        torch.cuda.synchronize()
        e_ms = replicas.max_over_ranks(ev2.elapsed_time(ev3), world, "cuda")
        return replicas.aggregate_gteps(world, n_e2e, E, e_ms)

    e2e_sync_value = timed_e2e(lambda i: eng.bfs(src_of(i), depth_out=host_bufs[0].array))
    # the pipelined call needs graph mode; the host-driven loop has the synchronous one only
    e2e_value = e2e_sync_value if args.host_loop else \
        timed_e2e(lambda i: eng.bfs_enqueue(src_of(i), host_bufs[i & 1].array))

    # roofline of the dominant kernel from per-level device times over every
    # source (separate, untimed pass)
    per_dir = {0: [0, 0.0, 0], 1: [0, 0.0, 0]}  # alg bytes, ms, launches
    eng_h = S.Engine(g, device=local_rank, stream=stream.cuda_stream, use_graph=2)  # per-level CUDA events
    for s in srcs:
        eng_h.bfs(s)
        for t in eng_h.trace():
            a = per_dir[t["direction"]]
            a[0] += t["alg_bytes"]
            a[1] += t["ms"]
            a[2] += 1
    dom = max(per_dir, key=lambda d: per_dir[d][1])
    alg, dms, nl = per_dir[dom]
    peak, peak_kind = hbm_peak()
    achieved = (alg / nl) / (dms / nl / 1e3) / 1e9 if nl and dms > 0 else None
    roof = {"bound": "hbm", "kernel": "k_pull" if dom == 1 else "k_push(+k_push_giant)",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "frac_of_nominal": achieved / NOMINAL_HBM_GBS if achieved else None,  # B200 HBM3e, 8 TB/s
            "alg_bytes_rule": "push: 12 B per frontier vertex + 4 B per edge; pull: 12 B per unvisited vertex + "
                              "4 B per in-edge inspected; each level V/8 B of bitmap + 4 B per discovered vertex; "
                              "frontier/visited probes not counted (bitmaps of %.1f MB, L2-resident)"
                              % (csr.V / 8 / 1e6),
            # DRAM read+write per k_pull launch, ncu over every k_pull launch of the same
            # command with --host-loop (K_PULL_TRAFFIC_BYTES)
            "traffic": K_PULL_TRAFFIC_BYTES if dom == 1 and args.scale == 24 else None,
            "launches_sampled": nl, "alg_bytes_per_launch": alg / nl if nl else None,
            "share_of_level_time": dms / (per_dir[0][1] + per_dir[1][1])}

    line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded RMAT)",
            "config": config_dict(V, E, args.scale, len(srcs)),
            "parallelism": f"replicas x{world}", "graph_gen_s": round(gen_s, 1), "parity": parity,
            "autotune": tune,
            "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 4, "d2h_bytes_per_step": V * 4,
                    "api": "scaph_bfs (one step at a time)" if args.host_loop else
                           "scaph_bfs_enqueue (pipelined, page-locked host output)",
                    "sync_value": e2e_sync_value, "sync_api": "scaph_bfs (one step at a time)"},
            "gpu_launches": launches, "roofline": roof, "clocks": clk,
            "graph500_gteps_median": statistics.median(g500)}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(csr, srcs, args.cpu_seconds)
        line["cpu_baseline_openmp"] = line["cpu_baseline"].pop("openmp")
    for b in host_bufs:
        b.close()
    eng_h.close()
    eng.close()
    if rank == 0 and world == 1 and not args.no_extras:
        # each configuration in its own process: a fresh host heap for the big
        # generated graphs, and a failure there cannot take the headline down
        extras = {}
        names = ["pcie", "config1", "config4a_batched", "config4b_mixed", "config2_learned", "config3_learned"]
        if not args.no_config5:
            names.append("config5_ooc_batched")
        for name in names:
            try:
                r = subprocess.run([sys.executable, os.path.abspath(__file__), "--only-extra", name],
                                   capture_output=True, text=True, timeout=1200)
                last = [l for l in r.stdout.splitlines() if l.startswith("{")]
                extras[name] = json.loads(last[-1]) if r.returncode == 0 and last else \
                    {"error": f"exit {r.returncode}: {r.stderr[-400:]}"}
            except Exception as exc:  # report, keep the headline line
                extras[name] = {"error": f"{type(exc).__name__}: {exc}"}
            print(f"[bench] {name}: {json.dumps(extras[name])[:300]}", file=sys.stderr, flush=True)
        line["extras"] = extras
        line["learned_batched_vs_plain"] = learned_batched_vs_plain(extras)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


EXTRAS = {
    "pcie": lambda st: extra_pcie(st),
    "config1": lambda st: extra_config1(),
    "config4a_batched": lambda st: extra_config4a(st),
    "config4b_mixed": lambda st: extra_config4b(st),
    "config3_learned": lambda st: extra_config3(),
    "config2_learned": lambda st: extra_config2_learned(st),
    "config5_ooc_batched": lambda st: extra_config5(st),
}


def run_extra(name):
    import torch

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    print(json.dumps(EXTRAS[name](stream)), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.only_extra:
        run_extra(args.only_extra)
        return
    if args.impl == "reference":
        run_reference(args, world)
    else:
        run_ours(args, world)


if __name__ == "__main__":
    main()
