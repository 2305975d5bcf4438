"""Learned BFS scheduler: training data, labels, training, evaluation.

The network (scaph_b200.Mlp, GPU kernels in csrc/mlp.cu) sees, before every
level, the feature row the engine computes (16 globals + the frontier's
share of every out-edge page; layout in include/scaph/scaph.h) and predicts

  * output 0: push (< 0) or pull (> 0) for the level, and
  * outputs 1..P: whether out-page p holds frontier vertices at the NEXT
    level (used to prefetch pages while the level runs).

Training data comes from the plain engine itself: the graph is traversed
resident in HBM with dual timing (every level run both ways from the same
state), which gives the kernel time of either direction at every level.
Direction labels then come from an out-of-core cost model: for every
direction sequence with at most two switches (push..push pull..pull push..),
total cost = kernel times + page traffic of a cold LRU page pool of the
engine's size (pages a push needs: out-pages holding the frontier; a pull:
in-pages holding unvisited vertices) at the PCIe bandwidth; the cheapest
sequence labels the levels.  The residency and previous-direction features
of the training rows are recomputed along that sequence.  The alpha/beta
switch stays the fallback and the yardstick of its per-level time and page
traffic: the network only picks directions and prefetches pages, the
depths never change.
"""
from __future__ import annotations

import time

from dataclasses import dataclass

import numpy as np

from . import DIR_LEARNED, Engine, Mlp, PagedGraph

G = 16  # SCAPH_SCHED_GLOBALS


@dataclass
class Trace:
    src: int
    feats: np.ndarray        # levels x (G + P): rows as the engine computed them
    push_ms: np.ndarray      # levels
    pull_ms: np.ndarray      # levels
    nf: np.ndarray           # frontier size per level
    mf: np.ndarray           # frontier out-edges per level
    mu: np.ndarray           # unexplored edges per level
    out_need: list           # out-pages a push would read, per level
    in_need: list            # in-pages a pull would read, per level
    out_datas: list          # their active words sum(deg+3), per level
    in_datas: list
    next_active: np.ndarray  # levels x P: out-page holds frontier at the next level


def collect(g: PagedGraph, gt: PagedGraph | None, sources, **engine_kw) -> list[Trace]:
    """Dual-timed, feature-recording plain runs (graph resident in HBM)."""
    eng = Engine(g, gt, use_graph=2, record_features=1, dual_timing=1, **engine_kw)
    npi = (gt or g).npages
    P = g.npages
    out = []
    for s in sources:
        eng.bfs(int(s))
        tr = eng.trace()
        F = eng.features()
        L = len(tr)
        nxt = np.zeros((L, P), np.float32)
        out_need, out_datas = [], []
        deg_src = int(g.degree()[int(s)])
        for lvl in range(L):
            hn, _ = eng.page_hist(lvl + 1)  # frontier of level lvl+1
            nxt[lvl] = hn > 0
            if lvl == 0:
                pages = np.flatnonzero(F[0, G:] > 0)
                out_need.append(pages)
                out_datas.append(np.full(len(pages), deg_src + 3, np.int64))
            else:
                hp, hd = eng.page_hist(lvl)
                pages = np.flatnonzero(hp > 0)
                out_need.append(pages)
                out_datas.append(hd[pages].astype(np.int64))
        in_need, in_datas = [], []
        for lvl in range(L):
            c, d = eng.pull_pages(lvl, npi)
            pages = np.flatnonzero(c > 0)
            in_need.append(pages)
            in_datas.append(d[pages].astype(np.int64))
        push = np.array([t["push_ms"] for t in tr])
        pull = np.array([t["pull_ms"] if lvl > 0 else np.inf for lvl, t in enumerate(tr)])
        out.append(Trace(int(s), F, push, pull, np.array([t["frontier"] for t in tr], np.float64),
                         np.array([t["frontier_edges"] for t in tr], np.float64),
                         np.array([t["unvisited_edges"] for t in tr], np.float64), out_need, in_need, out_datas,
                         in_datas, nxt))
    eng.close()
    return out


def collect_ms(g: PagedGraph, gt: PagedGraph | None, batches, depth_ptr: int | None = None,
               **engine_kw) -> list[np.ndarray]:
    """Feature rows of multi-source traversals (one array of levels x (G+P)
    per batch of sources): the union of the batch's frontiers, counted per
    out-page.  They teach the page outputs what a batched frontier spreads
    to; their direction output is not trained (the multi-source kernels'
    costs differ from the single-source labels).  depth_ptr: a device
    buffer of len(batch) * V words for the depths (else host memory)."""
    eng = Engine(g, gt, record_features=1, **engine_kw)
    out = []
    for b in batches:
        b = [int(x) for x in b]
        if depth_ptr is None:
            eng.msbfs(b)
        else:
            eng.msbfs_device(b, depth_ptr)
        out.append(eng.features())
    eng.close()
    return out


def ms_dataset(rows_list, n_out: int, w_page=0.5):
    """Training rows of multi-source traces: page labels are the next row's
    frontier pages (none after the last level); direction weight 0."""
    Xs, Ts, Ws = [], [], []
    for F in rows_list:
        L = len(F)
        nxt = np.zeros((L, n_out), np.float32)
        if L > 1:
            nxt[:-1] = F[1:, G:] > 0
        T = np.concatenate([np.zeros((L, 1), np.float32), nxt], axis=1)
        W = np.zeros_like(T)
        W[:, 1:] = w_page / n_out
        Xs.append(F.astype(np.float32))
        Ts.append(T)
        Ws.append(W)
    return np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ws)


def alpha_beta(cur, nf, prev_nf, mf, mu, V, alpha=14.0, beta=96.0) -> int:
    """Beamer's rule, as the engine applies it (0 push, 1 pull)."""
    if cur == 0:
        return 1 if mf > mu / alpha else 0
    return 0 if (nf < V / beta and nf < prev_nf) else 1


class PoolSim:
    """LRU page pool shared by out- and in-pages (cold at start)."""

    def __init__(self, nslots: int):
        self.nslots = nslots
        self.slot = {}  # (graph, page) -> last use
        self.clock = 0

    def resident(self, gid, pages):
        if len(pages) == 0:
            return 1.0
        return float(np.mean([(gid, int(p)) in self.slot for p in pages]))

    def resident_all(self, gid, npages):
        return sum(1 for (g, _) in self.slot if g == gid) / max(1, npages)

    def touch(self, gid, pages) -> int:
        """Makes `pages` resident; returns how many had to be fetched."""
        self.clock += 1
        fetched = 0
        need = {(gid, int(p)) for p in pages}
        for key in need:
            if key in self.slot:
                self.slot[key] = self.clock
                continue
            if len(self.slot) >= self.nslots:
                victims = [k for k in self.slot if k not in need]
                if victims:
                    del self.slot[min(victims, key=lambda k: self.slot[k])]
                else:
                    fetched += 1  # streamed through without staying
                    continue
            self.slot[key] = self.clock
            fetched += 1
        return fetched


def sequences(L: int):
    """Direction sequences (level 0 push) with at most two switches:
    push [1,i) pull [i,j) push [j,L)."""
    for i in range(1, L + 1):
        for j in range(i, L + 1):
            yield [0] + [0 if (lvl < i or lvl >= j) else 1 for lvl in range(1, L)]


def label(tr: Trace, nslots: int, page_ms: float, V: int, n_out: int, n_in: int, symmetric: bool,
          alpha=14.0, beta=96.0, resident=False, zc_words=None, page_words=None):
    """Cheapest sequence under the cost model; returns (dirs, feature rows
    recomputed along it, its cost, alpha/beta's cost).  resident=True: the
    graph is all in HBM (no page traffic, residency features 1).  Pages whose
    active words are at most zc_words (the engine's compact threshold) are
    read zero-copy at their byte cost instead of being copied, as the engine
    does."""
    L = len(tr.push_ms)
    gin = 0 if symmetric else 1
    if resident:
        page_ms = 0.0
        nslots = n_out + n_in
    words_ms = page_ms / page_words if page_words else 0.0

    def need(gid, pages, datas, sim):
        """Cost of one level's pages: zero-copy the sparse non-resident ones."""
        big, zc = [], 0
        for p, d in zip(pages, datas):
            if zc_words is not None and d <= zc_words and (gid, int(p)) not in sim.slot:
                zc += int(d)
            else:
                big.append(p)
        return sim.touch(gid, big) * page_ms + zc * words_ms

    def cost(seq, want_rows=False):
        sim = PoolSim(nslots)
        if resident:
            for gid, npg in ((0, n_out), (gin, n_in)):
                sim.touch(gid, range(npg))
        total = 0.0
        rows = tr.feats.copy() if want_rows else None
        for lvl in range(L):
            d = seq[lvl]
            if want_rows:
                prev = seq[lvl - 1] if lvl else 0
                rows[lvl, 9] = prev
                rows[lvl, 10] = sim.resident_all(0, n_out)
                rows[lvl, 11] = sim.resident_all(gin, n_in)
                rows[lvl, 12] = sim.resident(0, tr.out_need[lvl])
                rows[lvl, 13] = sim.resident(gin, tr.in_need[lvl])
                rows[lvl, 14] = 0 if lvl == 0 else alpha_beta(prev, tr.nf[lvl], tr.nf[lvl - 1], tr.mf[lvl],
                                                             tr.mu[lvl], V, alpha, beta)
            k = tr.push_ms[lvl] if d == 0 else tr.pull_ms[lvl]
            if d == 0:
                total += k + need(0, tr.out_need[lvl], tr.out_datas[lvl], sim)
            else:
                total += k + need(gin, tr.in_need[lvl], tr.in_datas[lvl], sim)
        return total, rows

    # alpha/beta's own sequence
    ab = [0]
    for lvl in range(1, L):
        ab.append(alpha_beta(ab[-1], tr.nf[lvl], tr.nf[lvl - 1], tr.mf[lvl], tr.mu[lvl], V, alpha, beta))
    ab_cost, _ = cost(ab)
    best, best_cost = ab, ab_cost
    for seq in sequences(L):
        c, _ = cost(seq)
        if c < best_cost - 1e-9:
            best, best_cost = seq, c
    _, rows = cost(best, want_rows=True)
    return np.array(best, np.float32), rows, best_cost, ab_cost


def dataset(traces, nslots, page_ms, V, n_out, n_in, symmetric, w_dir=1.0, w_page=0.5, zc_words=None,
            page_words=None):
    """Training rows: the direction labels are the kernel-time optimum of
    the resident graph (the engine adds the exact page-traffic cost of each
    direction itself when it runs out of core)."""
    Xs, Ts, Ws = [], [], []
    for tr in traces:
        for resident in (True,):
            dirs, rows, _, _ = label(tr, nslots, page_ms, V, n_out, n_in, symmetric, resident=resident,
                                     zc_words=zc_words, page_words=page_words)
            T = np.concatenate([dirs[:, None], tr.next_active], axis=1)
            W = np.zeros_like(T)
            W[1:, 0] = w_dir  # level 0 is always push
            W[:, 1:] = w_page / n_out
            Xs.append(rows)
            Ts.append(T)
            Ws.append(W)
    X, T, W = np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ws)
    W /= len(X)
    return X.astype(np.float32), T.astype(np.float32), W.astype(np.float32)


def train(traces, g: PagedGraph, gt: PagedGraph | None, nslots: int, page_ms: float, epochs=300, lr=3e-3,
          seed=7, device=0, compact_threshold=3, ms_rows=None) -> tuple[Mlp, dict]:
    """Trains the network on the single-source traces (direction and page
    labels) and, optionally, multi-source feature rows (collect_ms: page
    labels only)."""
    n_out, n_in = g.npages, (gt or g).npages
    zc_words = compact_threshold * (g.pagesize // 32)
    X, T, W = dataset(traces, nslots, page_ms, g.V, n_out, n_in, gt is None, zc_words=zc_words,
                      page_words=g.pagesize)
    if ms_rows:
        Xm, Tm, Wm = ms_dataset(ms_rows, n_out)
        # dataset() normalised its weights by its row count; the same for these
        W = W * len(X)
        X, T, W = np.concatenate([X, Xm]), np.concatenate([T, Tm]), np.concatenate([W, Wm])
        W /= len(X)
    net = Mlp(G + n_out, 1 + n_out, seed=seed, device=device)
    loss0, _ = net.loss_grad(X, T, W)
    batch = min(256, len(X))
    t0 = time.perf_counter()
    loss = net.train(X, T, W, epochs=epochs, batch=batch, lr=lr, seed=seed)
    t1 = time.perf_counter()
    Y = net.forward(X)
    t2 = time.perf_counter()
    m = W[:, 0] > 0
    acc = float(((Y[m, 0] > 0) == (T[m, 0] > 0.5)).mean()) if m.any() else 1.0
    steps = epochs * -(-len(X) // batch)
    # device time of the network's kernels (CUDA events), beside the host
    # wall clock of the training call (which copies every minibatch in)
    dev = net.time(n=batch, reps=20)
    return net, {"rows": int(len(X)), "loss0": loss0, "loss": loss, "direction_accuracy": acc,
                 "train_steps": steps, "batch": batch, "device_us": dev,
                 "host_wall_us_per_train_step": (t1 - t0) * 1e6 / max(1, steps),
                 "host_wall_us_forward_call": (t2 - t1) * 1e6}


def held_out_accuracy(net: Mlp, traces, g: PagedGraph, gt: PagedGraph | None, nslots: int, page_ms: float,
                      compact_threshold=3, prefetch_logit=2.0) -> dict:
    """The trained network on traces it was not trained on: direction
    accuracy against the same labels (levels 1..), and the page prediction
    as the engine uses it (prefetch where the logit exceeds prefetch_logit):
    precision and recall against the pages that really hold the next
    level's frontier."""
    n_out, n_in = g.npages, (gt or g).npages
    X, T, W = dataset(traces, nslots, page_ms, g.V, n_out, n_in, gt is None,
                      zc_words=compact_threshold * (g.pagesize // 32), page_words=g.pagesize)
    Y = net.forward(X)
    m = W[:, 0] > 0
    dir_acc = float(((Y[m, 0] > 0) == (T[m, 0] > 0.5)).mean()) if m.any() else 1.0
    pred, true = Y[:, 1:] > prefetch_logit, T[:, 1:] > 0.5
    tp = int((pred & true).sum())
    return {"rows": int(len(X)), "direction_rows": int(m.sum()), "direction_accuracy": dir_acc,
            "prefetch_precision": tp / max(1, int(pred.sum())), "prefetch_recall": tp / max(1, int(true.sum())),
            "prefetch_logit": prefetch_logit}


def evaluate(g: PagedGraph, gt: PagedGraph | None, sources, net: Mlp | None, pool_bytes: int, cold=True,
             **engine_kw) -> dict:
    """Out-of-core runs of `sources`: alpha/beta + demand paging, or the learned
    scheduler (direction + prefetch).  Cold pool before every source."""
    eng = Engine(g, gt, pool_bytes=pool_bytes, direction=DIR_LEARNED if net is not None else 0, **engine_kw)
    if net is not None:
        eng.set_scheduler(net)
    ms, h2d, faults, pref, edges = 0.0, 0, 0, 0, 0
    depths = []
    for s in sources:
        if cold:
            eng.evict_all()
        d, _, st = eng.bfs(int(s))
        depths.append(d)
        ms += st.ms
        h2d += st.h2d_bytes
        faults += st.page_faults
        pref += st.prefetched
        edges += g.E
    eng.close()
    return {"ms": ms, "h2d_bytes": h2d, "page_faults": faults, "prefetched": pref,
            "gteps": edges / (ms / 1e3) / 1e9 if ms > 0 else 0.0, "depths": depths}
