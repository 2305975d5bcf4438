"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs, as the checker.  The engine (scaph_b200) never imports this module.

* liboracle.so      - bfs_oracle.c, the C restatement of the reference's
                      CPU BFS (app/bfs.cu:70-101) and helpers.
* _ref/libscaphref.so, _ref/pagegencsr, _ref/bin2ligra, _ref/bin2ligraweight,
  _ref/bin2totem    - the reference's own code compiled from its sources by
                      oracle/Makefile (only present where the reference tree
                      was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
# Root of the reference source tree where it is present (the recipes in
# oracle/Makefile and __graft_entry__.build() compile it from there); only
# build-and-compare tests read it, and they skip when it is absent.
REFERENCE_DIR = os.environ.get("SCAPH_REFERENCE", "/root/reference")
REF_SO = os.path.join(HERE, "_ref", "libscaphref.so")
REF_PAGEGEN = os.path.join(HERE, "_ref", "pagegencsr")
# the reference's CSR -> text converters (tools/bin2ligra.cpp, bin2ligraweight.cpp,
# bin2totem.cpp); bin2totemweight.cpp is not built: it reads E weights into a
# buffer of V+1 words (tools/bin2totemweight.cpp:94-96)
REF_EXPORTERS = {k: os.path.join(HERE, "_ref", k) for k in ("bin2ligra", "bin2ligraweight", "bin2totem")}

_o = None
_r = None


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def olib() -> C.CDLL:
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        L = C.CDLL(ORACLE_SO)
        vp, u32, i64, i32 = C.c_void_p, C.c_uint32, C.c_int64, C.c_int
        L.oracle_bfs.argtypes = [u32, vp, vp, u32, u32, vp]
        L.oracle_bfs.restype = i64
        L.oracle_bfs_omp.argtypes = [u32, vp, vp, u32, u32, vp, i32]
        L.oracle_bfs_omp.restype = i64
        L.oracle_bfs_paged.argtypes = [u32, i64, vp, vp, i32, u32, u32, vp]
        L.oracle_bfs_paged.restype = i64
        L.oracle_validate_tree.argtypes = [u32, vp, vp, u32, u32, vp, vp, C.POINTER(u32)]
        L.oracle_validate_tree.restype = i32
        L.oracle_page_stats.argtypes = [i64, vp, vp, vp, i32, vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.oracle_page_stats.restype = None
        L.oracle_compact_page.argtypes = [vp, vp, vp, u32, u32, u32, i32]
        L.oracle_compact_page.restype = u32
        L.oracle_max_zero_run.argtypes = [u32]
        L.oracle_max_zero_run.restype = i32
        L.oracle_fit_zero_run.argtypes = [u32, i32]
        L.oracle_fit_zero_run.restype = i32
        L.oracle_set_run.argtypes = [u32, i32, i32, i32]
        L.oracle_set_run.restype = u32
        L.oracle_hook_fixpoint.argtypes = [u32, vp, vp, vp, i32, vp, vp]
        L.oracle_hook_fixpoint.restype = i64
        L.oracle_sssp_dijkstra.argtypes = [u32, vp, vp, vp, u32, u32, vp]
        L.oracle_sssp_dijkstra.restype = i32
        L.oracle_min_reaching_id.argtypes = [u32, vp, vp, vp]
        L.oracle_min_reaching_id.restype = i32
        L.oracle_gen_rmat.argtypes = [i32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, i32, vp,
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
        L.oracle_gen_rmat.restype = i32
        L.oracle_free.argtypes = [vp]
        L.oracle_free.restype = None
        _o = L
    return _o


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def rlib() -> C.CDLL:
    global _r
    if _r is None:
        L = C.CDLL(REF_SO)
        vp, u32, i32 = C.c_void_p, C.c_uint, C.c_int
        L.ref_bfs_check.argtypes = [u32, vp, vp, u32, vp, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
        L.ref_bfs_check.restype = i32
        L.ref_compress_stat.argtypes = [vp, vp, vp, u32, u32, u32]
        L.ref_compress_stat.restype = u32
        L.ref_max_zero_run.argtypes = [i32]
        L.ref_max_zero_run.restype = i32
        L.ref_fit_zero_run.argtypes = [i32, i32]
        L.ref_fit_zero_run.restype = i32
        L.ref_set_run.argtypes = [i32, i32, i32, i32]
        L.ref_set_run.restype = i32
        _r = L
    return _r


def _csr(idx, ngh):
    return np.ascontiguousarray(idx, np.uint64), np.ascontiguousarray(ngh, np.uint32)


def gen_rmat(scale: int, edgefactor: float, a: float, b: float, c: float, seed: int, scramble: bool = True):
    """The seeded RMAT graph of scaph_gen_rmat, generated without the
    product library (gen_oracle.c): (idx uint64[V+1], ngh uint32[E])."""
    V = 1 << scale
    idx = np.empty(V + 1, np.uint64)
    ptr, E = C.c_void_p(), C.c_uint64()
    if olib().oracle_gen_rmat(scale, edgefactor, a, b, c, seed, 1 if scramble else 0, _p(idx), C.byref(ptr),
                              C.byref(E)) != 0:
        raise MemoryError("oracle_gen_rmat failed")
    try:
        ngh = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), shape=(max(1, E.value),))[:E.value].copy()
    finally:
        olib().oracle_free(ptr)
    return idx, ngh


def bfs(idx, ngh, src: int, unreached: int = 0xFFFFFFFF) -> np.ndarray:
    """Single-threaded level-synchronous BFS (app/bfs.cu:70-101)."""
    idx, ngh = _csr(idx, ngh)
    V = len(idx) - 1
    d = np.empty(V, np.uint32)
    if olib().oracle_bfs(V, _p(idx), _p(ngh), src, unreached, _p(d)) < 0:
        raise ValueError("oracle_bfs: bad input")
    return d


def bfs_omp(idx, ngh, src: int, unreached: int = 0xFFFFFFFF, threads: int = 0) -> np.ndarray:
    idx, ngh = _csr(idx, ngh)
    V = len(idx) - 1
    d = np.empty(V, np.uint32)
    if olib().oracle_bfs_omp(V, _p(idx), _p(ngh), src, unreached, _p(d), threads) < 0:
        raise ValueError("oracle_bfs_omp: bad input")
    return d


def bfs_paged(V: int, page_list: np.ndarray, pages: list, src: int, unreached: int = 0xFFFFFFFF,
              weighted: bool = False) -> np.ndarray:
    pl = np.ascontiguousarray(page_list, np.uint32)
    ptrs = (C.c_void_p * len(pages))(*[p.ctypes.data for p in pages])
    d = np.empty(V, np.uint32)
    if olib().oracle_bfs_paged(V, len(pages), _p(pl), ptrs, int(weighted), src, unreached, _p(d)) < 0:
        raise ValueError("oracle_bfs_paged: bad input")
    return d


def validate_tree(idx, ngh, src: int, depth: np.ndarray, parent: np.ndarray, unreached: int = 0xFFFFFFFF):
    """Returns (code, vertex): code 0 = valid BFS tree."""
    idx, ngh = _csr(idx, ngh)
    depth = np.ascontiguousarray(depth, np.uint32)
    parent = np.ascontiguousarray(parent, np.uint32)
    bad = C.c_uint32(0)
    rc = olib().oracle_validate_tree(len(idx) - 1, _p(idx), _p(ngh), src, unreached, _p(depth), _p(parent),
                                     C.byref(bad))
    return rc, bad.value


def page_stats(page_list, stat, degree, weighted=False):
    pl = np.ascontiguousarray(page_list, np.uint32)
    stat = np.ascontiguousarray(stat, np.uint8)
    degree = np.ascontiguousarray(degree, np.uint32)
    n = len(pl)
    nodes = np.zeros(n, np.uint32)
    datas = np.zeros(n, np.uint32)
    tn, td = C.c_int64(), C.c_int64()
    olib().oracle_page_stats(n, _p(pl), _p(stat), _p(degree), int(weighted), _p(nodes), _p(datas),
                             C.byref(tn), C.byref(td))
    return nodes, datas, tn.value, td.value


def compact_page(page_src, stat, left, srcnodenum, dstnodenum, weighted=False, out_words=None):
    src = np.ascontiguousarray(page_src, np.uint32)
    stat = np.ascontiguousarray(stat, np.uint8)
    dst = np.zeros(out_words or len(src), np.uint32)
    n = olib().oracle_compact_page(_p(src), _p(dst), _p(stat), left, srcnodenum, dstnodenum, int(weighted))
    return dst, n


def ref_bfs_check(idx32, ngh, src: int, values: np.ndarray):
    """Runs the reference's own bfs::check; returns (mismatches, seconds)."""
    idx32 = np.ascontiguousarray(idx32, np.uint32)
    ngh = np.ascontiguousarray(ngh, np.uint32)
    values = np.ascontiguousarray(values, np.uint32).copy()
    err, sec = C.c_longlong(), C.c_double()
    rc = rlib().ref_bfs_check(len(idx32) - 1, _p(idx32), _p(ngh), src, _p(values), C.byref(err), C.byref(sec))
    if rc != 0:
        raise RuntimeError("ref_bfs_check: could not parse the reference output")
    return err.value, sec.value


HOOK_APPS = {"bfs": 0, "sssp": 1, "wcc": 2}


def hook_fixpoint(idx, ngh, app: str, value, active, wgh=None) -> np.ndarray:
    """Fixed point of an app's hooks (bfs / sssp / wcc) from the initial
    values and active flags gpu_init() would leave; returns the values."""
    idx, ngh = _csr(idx, ngh)
    value = np.ascontiguousarray(value, np.uint32).copy()
    active = np.ascontiguousarray(active, np.uint8)
    w = None if wgh is None else np.ascontiguousarray(wgh, np.uint32)
    n = olib().oracle_hook_fixpoint(len(idx) - 1, _p(idx), _p(ngh), _p(w), HOOK_APPS[app], _p(value), _p(active))
    if n < 0:
        raise ValueError("oracle_hook_fixpoint: bad arguments")
    return value


def sssp_dijkstra(idx, ngh, wgh, src: int, far: int = 0x7FFFFFFF) -> np.ndarray:
    idx, ngh = _csr(idx, ngh)
    wgh = np.ascontiguousarray(wgh, np.uint32)
    out = np.zeros(len(idx) - 1, np.uint32)
    if olib().oracle_sssp_dijkstra(len(idx) - 1, _p(idx), _p(ngh), _p(wgh), src, far, _p(out)) != 0:
        raise ValueError("oracle_sssp_dijkstra failed")
    return out


def min_reaching_id(idx, ngh) -> np.ndarray:
    idx, ngh = _csr(idx, ngh)
    out = np.zeros(len(idx) - 1, np.uint32)
    if olib().oracle_min_reaching_id(len(idx) - 1, _p(idx), _p(ngh), _p(out)) != 0:
        raise ValueError("oracle_min_reaching_id failed")
    return out


def export_text(idx32, ngh, wgh, kind: str) -> bytes:
    """The reference converters' text formats, restated (small graphs only):
    "ligra" / "ligra.weight" (tools/bin2ligra.cpp:92-104,
    tools/bin2ligraweight.cpp:99-115): a header line, V, E, then the V
    offsets idx[0..V-1], the E neighbours (and the E weights), one per line;
    "totem" / "weight.totem" (tools/bin2totem.cpp:92-104,
    tools/bin2totemweight.cpp:99-111): "#Nodes: V", "#Edges: E",
    "#Undirected", then one "src<TAB>dst[<TAB>weight]" line per edge."""
    V, E = len(idx32) - 1, len(ngh)
    if wgh is None:  # the weight file of an unweighted graph holds zeros
        wgh = np.zeros(E, np.uint32)
    lines = []
    if kind in ("ligra", "ligra.weight"):
        lines.append("WeightedAdjacencyGraph" if kind == "ligra.weight" else "AdjacencyGraph")
        lines += [str(V), str(E)]
        lines += [str(int(x)) for x in idx32[:V]]
        lines += [str(int(x)) for x in ngh]
        if kind == "ligra.weight":
            lines += [str(int(x)) for x in wgh]
    else:
        lines += [f"#Nodes: {V}", f"#Edges: {E}", "#Undirected"]
        for v in range(V):
            for e in range(int(idx32[v]), int(idx32[v + 1])):
                if kind == "weight.totem":
                    lines.append(f"{v}\t{int(ngh[e])}\t{int(wgh[e])}")
                else:
                    lines.append(f"{v}\t{int(ngh[e])}")
    return ("\n".join(lines) + "\n").encode()


def pagerank(idx, ngh, iters: int = 20, damping: float = 0.85) -> np.ndarray:
    """PageRank by power iteration in float64 (the rule scaph_b200/apps/pr
    applies in float32): rank'(v) = (1-d)/V + d * (sum over edges u->v of
    rank(u)/outdeg(u) + (rank of vertices without out-edges)/V), from the
    uniform vector.  The reference has no working PageRank to restate
    (app/pr.cu does not build)."""
    idx, ngh = _csr(idx, ngh)
    V = len(idx) - 1
    deg = np.diff(idx).astype(np.float64)
    src = np.repeat(np.arange(V), np.diff(idx).astype(np.int64))
    rank = np.full(V, 1.0 / V)
    for _ in range(iters):
        contrib = np.where(deg > 0, rank / np.maximum(deg, 1.0), 0.0)
        dangling = rank[deg == 0].sum()
        acc = np.bincount(ngh, weights=contrib[src], minlength=V)
        rank = (1.0 - damping) / V + damping * (acc + dangling / V)
    return rank
