"""scaph_b200 - the Scaph BFS hot path rebuilt for B200 (sm_100a).

Python mirror of the C ABI in include/scaph/scaph.h (libscaph.so, built
in-tree by scaph_b200/Makefile).  The engine itself is C++/CUDA; this module
only marshals arguments with ctypes and numpy.  There is no CPU fallback: if
libscaph.so is missing, importing the engine raises ScaphError.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# SCAPH_LIB may point at another build of the same library (e.g. a variant
# compiled with different tile parameters).
LIB_PATH = os.environ.get("SCAPH_LIB", os.path.join(_HERE, "libscaph.so"))

# status codes (include/scaph/scaph.h)
OK, EINVAL, EIO, ENOMEM, ECUDA, EFORMAT, ETIMEOUT, EUNSUPPORTED, EDEVICE = 0, -1, -2, -3, -4, -5, -6, -7, -8
DIR_ALPHABETA, DIR_PUSH, DIR_PULL, DIR_LEARNED = 0, 1, 2, 3
UNREACHED = 0xFFFFFFFF
REF_UNREACHED = 63  # MAXDEPTH of the reference BFS app (app/bfs.cu:18)
NOALLOC_SYMMETRIC = 1  # scaph_bfs_page_noalloc: the page is symmetric, pull levels allowed
# text exports of <prefix>_csr.* (scaph_csr_export): kind -> file written
EXPORT_LIGRA, EXPORT_LIGRA_WEIGHT, EXPORT_TOTEM, EXPORT_TOTEM_WEIGHT = 1, 2, 3, 4
EXPORT_SUFFIX = {EXPORT_LIGRA: ".ligra", EXPORT_LIGRA_WEIGHT: ".ligra.weight", EXPORT_TOTEM: ".totem",
                 EXPORT_TOTEM_WEIGHT: "weight.totem"}


class ScaphError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"scaph error {code}: {msg}")
        self.code = code


class _Csr(C.Structure):
    _fields_ = [("V", C.c_uint32), ("E", C.c_uint64), ("idx", C.POINTER(C.c_uint64)),
                ("ngh", C.POINTER(C.c_uint32)), ("wgh", C.POINTER(C.c_uint32))]


class _GraphInfo(C.Structure):
    _fields_ = [("pagesize", C.c_uint32), ("V", C.c_uint32), ("E", C.c_uint64),
                ("npages", C.c_int32), ("weighted", C.c_int32)]


class _Config(C.Structure):
    _fields_ = [("pool_bytes", C.c_int64), ("unreached", C.c_uint32), ("direction", C.c_int32),
                ("alpha", C.c_float), ("beta", C.c_float), ("block_size", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("copy_streams", C.c_int32), ("prefetch", C.c_int32),
                ("compact_threshold", C.c_int32), ("use_graph", C.c_int32), ("device", C.c_int32),
                ("stream", C.c_void_p), ("record_features", C.c_int32), ("dual_timing", C.c_int32),
                ("link_gbs", C.c_float), ("giant_edges", C.c_int32), ("pull_gather_ratio", C.c_int32),
                ("ms_compact_l2_div", C.c_int32), ("ms_compact_min_deg", C.c_int32), ("pull_warp", C.c_int32),
                ("push_defer_edges", C.c_int64), ("pull_records", C.c_int32), ("pull_rows", C.c_int32),
                ("push_sparse_ratio", C.c_int32), ("pull_runs", C.c_int32)]


class _Stats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("push_levels", C.c_int32), ("pull_levels", C.c_int32),
                ("_pad", C.c_int32), ("reached", C.c_uint64), ("reached_edges", C.c_uint64),
                ("edges_inspected", C.c_uint64), ("alg_bytes", C.c_uint64), ("h2d_bytes", C.c_uint64),
                ("zc_bytes", C.c_uint64), ("page_faults", C.c_uint64), ("prefetched", C.c_uint64),
                ("launches", C.c_uint64), ("ms", C.c_double), ("pcie_alg_bytes", C.c_uint64)]


class _Query(C.Structure):
    _fields_ = [("graph", C.c_uint32), ("source", C.c_uint32)]


class _BatchParams(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("ctas_per_sm", C.c_int32), ("alpha", C.c_float), ("beta", C.c_float),
                ("_reserved", C.c_int32)]


class _Trace(C.Structure):
    _fields_ = [("level", C.c_int32), ("direction", C.c_int32), ("frontier", C.c_uint64),
                ("frontier_edges", C.c_uint64), ("unvisited", C.c_uint64), ("unvisited_edges", C.c_uint64),
                ("next", C.c_uint64), ("edges_inspected", C.c_uint64), ("alg_bytes", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("ms", C.c_double), ("push_ms", C.c_double), ("pull_ms", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """Loads libscaph.so (once).  Raises ScaphError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ScaphError(EUNSUPPORTED, f"{LIB_PATH} not built (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P, u32, u64, i32, vp = C.POINTER, C.c_uint32, C.c_uint64, C.c_int, C.c_void_p
    sig = {
        "scaph_last_error": ([], C.c_char_p),
        "scaph_version": ([], C.c_char_p),
        "scaph_gen_rmat": ([i32, C.c_double, C.c_double, C.c_double, C.c_double, u64, i32, P(_Csr)], i32),
        "scaph_gen_powerlaw": ([u32, u64, C.c_double, u32, u64, P(_Csr)], i32),
        "scaph_gen_web": ([u32, u64, C.c_double, u32, u32, C.c_double, u64, P(_Csr)], i32),
        "scaph_csr_transpose": ([P(_Csr), P(_Csr)], i32),
        "scaph_csr_from_arrays": ([u32, u64, vp, vp, vp, P(_Csr)], i32),
        "scaph_csr_free": ([P(_Csr)], None),
        "scaph_csr_write": ([C.c_char_p, P(_Csr)], i32),
        "scaph_csr_read": ([C.c_char_p, i32, P(_Csr)], i32),
        "scaph_pages_write": ([C.c_char_p, P(_Csr), u32, i32], i32),
        "scaph_pages_write_stream": ([C.c_char_p, C.c_char_p, u32, i32, i32, P(u32)], i32),
        "scaph_csr_export": ([C.c_char_p, i32], i32),
        "scaph_graph_open": ([C.c_char_p, i32, P(vp)], i32),
        "scaph_graph_from_csr": ([P(_Csr), u32, i32, P(vp)], i32),
        "scaph_graph_get_info": ([vp, P(_GraphInfo)], i32),
        "scaph_graph_page": ([vp, i32], P(u32)),
        "scaph_graph_page_list": ([vp], P(u32)),
        "scaph_graph_degree": ([vp], P(u32)),
        "scaph_graph_close": ([vp], None),
        "scaph_graph_to_csr": ([vp, P(_Csr)], i32),
        "scaph_csr_symmetric": ([P(_Csr)], i32),
        "scaph_engine_create": ([vp, vp, P(_Config), P(vp)], i32),
        "scaph_engine_destroy": ([vp], i32),
        "scaph_bfs": ([vp, u32, vp, vp, i32, P(_Stats)], i32),
        "scaph_bfs_trace": ([vp, P(_Trace), i32], i32),
        "scaph_engine_sync": ([vp], i32),
        "scaph_bfs_enqueue": ([vp, u32, vp], i32),
        "scaph_engine_evict_all": ([vp], i32),
        "scaph_engine_tune": ([vp, P(_Config)], i32),
        "scaph_mlp_create": ([i32, i32, u64, i32, P(vp)], i32),
        "scaph_mlp_destroy": ([vp], None),
        "scaph_mlp_num_params": ([vp], C.c_size_t),
        "scaph_mlp_get_params": ([vp, vp, C.c_size_t], i32),
        "scaph_mlp_set_params": ([vp, vp, C.c_size_t], i32),
        "scaph_mlp_forward": ([vp, vp, i32, vp], i32),
        "scaph_mlp_loss_grad": ([vp, vp, vp, vp, i32, P(C.c_float), vp], i32),
        "scaph_mlp_adam_step": ([vp, vp, vp, vp, i32, C.c_float, P(C.c_float)], i32),
        "scaph_mlp_train": ([vp, vp, vp, vp, i32, i32, i32, C.c_float, u64, P(C.c_float)], i32),
        "scaph_mlp_save": ([vp, C.c_char_p], i32),
        "scaph_mlp_time": ([vp, i32, i32, vp], i32),
        "scaph_mlp_load": ([vp, C.c_char_p], i32),
        "scaph_engine_set_scheduler": ([vp, vp], i32),
        "scaph_bfs_features": ([vp, vp, i32, P(i32)], i32),
        "scaph_bfs_pull_pages": ([vp, i32, vp, vp, i32], i32),
        "scaph_msbfs": ([vp, vp, i32, vp, i32, P(_Stats)], i32),
        "scaph_msbfs_trace": ([vp, P(_Trace), i32], i32),
        "scaph_bfs_page_hist": ([vp, i32, vp, vp, i32], i32),
        "scaph_batch_create": ([vp, i32, vp, u32, P(_Config), P(vp)], i32),
        "scaph_batch_destroy": ([vp], i32),
        "scaph_batch_graph_range": ([vp, i32, P(u32), P(u32)], i32),
        "scaph_batch_set_params": ([vp, P(_BatchParams)], i32),
        "scaph_batch_get_params": ([vp, P(_BatchParams)], i32),
        "scaph_batch_run": ([vp, vp, i32, vp, i32, P(_Stats)], i32),
        "scaph_batch_trace": ([vp, vp, i32], i32),
        "scaph_host_alloc": ([C.c_size_t], vp),
        "scaph_host_free": ([vp], None),
        "scaph_device_count": ([], i32),
        "scaph_fault_inject": ([C.c_char_p, i32, i32], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise ScaphError(rc, lib().scaph_last_error().decode())
    return rc


def _ptr(a: np.ndarray | None) -> C.c_void_p | None:
    return None if a is None else C.c_void_p(a.ctypes.data)


def fault_inject(site: str | None, skip: int = 0, count: int = 1) -> None:
    """Test hook (scaph_fault_inject): after `skip` further calls at `site`
    succeed, the next `count` fail as the CUDA runtime would report it;
    site None disarms every site."""
    _check(lib().scaph_fault_inject(site.encode() if site else None, skip, count))


def device_count() -> int:
    return lib().scaph_device_count()


class PinnedArray:
    """Page-locked host array (scaph_host_alloc) viewed as numpy; the target
    of asynchronous device->host copies (Engine.bfs_enqueue)."""

    def __init__(self, n: int, dtype=np.uint32):
        dt = np.dtype(dtype)
        self._p = lib().scaph_host_alloc(max(1, n) * dt.itemsize)
        if not self._p:
            raise ScaphError(ENOMEM, f"scaph_host_alloc({n * dt.itemsize}) failed")
        self.array = np.ctypeslib.as_array((C.c_uint8 * (max(1, n) * dt.itemsize)).from_address(self._p)).view(dt)[:n]

    def close(self) -> None:
        if self._p:
            self.array = None
            lib().scaph_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# flat CSR
# ---------------------------------------------------------------------------
class Csr:
    """Library-owned flat CSR (64-bit offsets, 32-bit neighbour ids)."""

    def __init__(self):
        self._c = _Csr()

    def __del__(self):
        if getattr(self, "_c", None) is not None and lib is not None:
            try:
                lib().scaph_csr_free(C.byref(self._c))
            except Exception:
                pass

    @property
    def V(self) -> int:
        return int(self._c.V)

    @property
    def E(self) -> int:
        return int(self._c.E)

    @property
    def idx(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._c.idx, shape=(self.V + 1,))

    @property
    def ngh(self) -> np.ndarray:
        if self.E == 0:
            return np.zeros(0, np.uint32)
        return np.ctypeslib.as_array(self._c.ngh, shape=(self.E,))

    @property
    def wgh(self) -> np.ndarray | None:
        if not self._c.wgh or self.E == 0:
            return None
        return np.ctypeslib.as_array(self._c.wgh, shape=(self.E,))

    def degree(self) -> np.ndarray:
        return np.diff(self.idx).astype(np.uint32)

    @classmethod
    def rmat(cls, scale: int, edgefactor: float = 16.0, a=0.57, b=0.19, c=0.19, seed: int = 1,
             scramble: bool = True) -> "Csr":
        g = cls()
        _check(lib().scaph_gen_rmat(scale, edgefactor, a, b, c, seed, int(scramble), C.byref(g._c)))
        return g

    @classmethod
    def powerlaw(cls, V: int, E: int, zipf_s: float = 1.9, max_degree: int = 0, seed: int = 1) -> "Csr":
        g = cls()
        _check(lib().scaph_gen_powerlaw(V, E, zipf_s, max_degree, seed, C.byref(g._c)))
        return g

    @classmethod
    def web(cls, V: int, E: int, s: float = 2.1, max_degree: int = 0, block: int = 4096,
            local_frac: float = 0.9, seed: int = 1) -> "Csr":
        g = cls()
        _check(lib().scaph_gen_web(V, E, s, max_degree, block, local_frac, seed, C.byref(g._c)))
        return g

    @classmethod
    def from_arrays(cls, idx, ngh, wgh=None) -> "Csr":
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        ngh = np.ascontiguousarray(ngh, dtype=np.uint32)
        w = None if wgh is None else np.ascontiguousarray(wgh, dtype=np.uint32)
        g = cls()
        _check(lib().scaph_csr_from_arrays(len(idx) - 1, len(ngh), _ptr(idx), _ptr(ngh), _ptr(w), C.byref(g._c)))
        return g

    @classmethod
    def read(cls, prefix: str, with_weights: bool = False) -> "Csr":
        g = cls()
        _check(lib().scaph_csr_read(prefix.encode(), int(with_weights), C.byref(g._c)))
        return g

    def symmetric(self) -> bool:
        """Whether every edge has its reverse (scaph_csr_symmetric)."""
        return _check(lib().scaph_csr_symmetric(C.byref(self._c))) == 1

    def transpose(self) -> "Csr":
        t = Csr()
        _check(lib().scaph_csr_transpose(C.byref(self._c), C.byref(t._c)))
        return t

    def write(self, prefix: str) -> None:
        _check(lib().scaph_csr_write(prefix.encode(), C.byref(self._c)))

    def write_pages(self, prefix: str, pagesize_words: int, weighted: bool = False) -> None:
        _check(lib().scaph_pages_write(prefix.encode(), C.byref(self._c), pagesize_words, int(weighted)))


def pages_write_stream(csr_prefix: str, out_prefix: str, pagesize_words: int, weighted: bool = False,
                       grow: bool = False) -> int:
    """Pages the flat CSR files <csr_prefix>_csr.* into <out_prefix>page*,
    reading the edges a page at a time (scaph_pages_write_stream); with grow
    a list longer than a page enlarges the page.  Returns the page size."""
    ps = C.c_uint32()
    _check(lib().scaph_pages_write_stream(csr_prefix.encode(), out_prefix.encode(), pagesize_words, int(weighted),
                                          1 if grow else 0, C.byref(ps)))
    return ps.value


def csr_export(prefix: str, kind: int) -> str:
    """Writes the text export `kind` (EXPORT_*) of the flat CSR files
    <prefix>_csr.* - what tools/bin2ligra, bin2ligraweight, bin2totem and
    bin2totemweight write - and returns the path written."""
    _check(lib().scaph_csr_export(prefix.encode(), kind))
    return prefix + EXPORT_SUFFIX[kind]


# ---------------------------------------------------------------------------
# paged CSR
# ---------------------------------------------------------------------------
class PagedGraph:
    """Host copy of a paged CSR (the reference's h_page / h_page_list)."""

    def __init__(self, handle: C.c_void_p, keep=None):
        self._h = handle
        self._keep = keep
        info = _GraphInfo()
        _check(lib().scaph_graph_get_info(self._h, C.byref(info)))
        self.pagesize, self.V, self.E = int(info.pagesize), int(info.V), int(info.E)
        self.npages, self.weighted = int(info.npages), bool(info.weighted)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().scaph_graph_close(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def open(cls, prefix: str, weighted: bool = False) -> "PagedGraph":
        h = C.c_void_p()
        _check(lib().scaph_graph_open(prefix.encode(), int(weighted), C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, csr: Csr, pagesize_words: int = 10 * 1024 * 1024, weighted: bool = False) -> "PagedGraph":
        h = C.c_void_p()
        _check(lib().scaph_graph_from_csr(C.byref(csr._c), pagesize_words, int(weighted), C.byref(h)))
        return cls(h)

    def page(self, p: int) -> np.ndarray:
        ptr = lib().scaph_graph_page(self._h, p)
        if not ptr:
            raise ScaphError(EINVAL, f"page {p} out of range")
        return np.ctypeslib.as_array(ptr, shape=(self.pagesize,))

    def page_list(self) -> np.ndarray:
        """Page{left,right,nodenum,edgenum}[npages] as an (npages, 4) uint32 array."""
        ptr = lib().scaph_graph_page_list(self._h)
        return np.ctypeslib.as_array(ptr, shape=(self.npages, 4))

    def degree(self) -> np.ndarray:
        return np.ctypeslib.as_array(lib().scaph_graph_degree(self._h), shape=(self.V,))

    def to_csr(self) -> Csr:
        """The flat CSR read back from the pages (scaph_graph_to_csr)."""
        c = Csr()
        _check(lib().scaph_graph_to_csr(self._h, C.byref(c._c)))
        return c


class Mlp:
    """The scheduler network (scaph_mlp_*): in -> 64 -> 64 -> out, BF16
    weights, FP32 accumulation, trained with the library's GPU kernels."""

    def __init__(self, in_dim: int, out_dim: int, seed: int = 1, device: int = 0):
        h = C.c_void_p()
        _check(lib().scaph_mlp_create(in_dim, out_dim, seed, device, C.byref(h)))
        self._h, self.in_dim, self.out_dim = h, in_dim, out_dim

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().scaph_mlp_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def num_params(self) -> int:
        return int(lib().scaph_mlp_num_params(self._h))

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        _check(lib().scaph_mlp_get_params(self._h, _ptr(out), out.size))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().scaph_mlp_set_params(self._h, _ptr(p), p.size))

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.zeros((X.shape[0], self.out_dim), np.float32)
        _check(lib().scaph_mlp_forward(self._h, _ptr(X), X.shape[0], _ptr(Y)))
        return Y

    def loss_grad(self, X, T, W):
        X, T, W = (np.ascontiguousarray(a, np.float32) for a in (X, T, W))
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float()
        _check(lib().scaph_mlp_loss_grad(self._h, _ptr(X), _ptr(T), _ptr(W), X.shape[0], C.byref(loss), _ptr(g)))
        return float(loss.value), g

    def train(self, X, T, W, epochs: int = 50, batch: int = 256, lr: float = 1e-3, seed: int = 1) -> float:
        X, T, W = (np.ascontiguousarray(a, np.float32) for a in (X, T, W))
        loss = C.c_float()
        _check(lib().scaph_mlp_train(self._h, _ptr(X), _ptr(T), _ptr(W), X.shape[0], epochs, batch, lr, seed,
                                     C.byref(loss)))
        return float(loss.value)

    def time(self, n: int = 256, reps: int = 20) -> dict:
        """Device microseconds (CUDA events) of a forward pass and a training
        step over n rows, and of the single-row inference kernel."""
        out = np.zeros(3, np.float32)
        _check(lib().scaph_mlp_time(self._h, n, reps, _ptr(out)))
        return {"forward_us": float(out[0]), "train_step_us": float(out[1]), "infer1_us": float(out[2]), "rows": n}

    def save(self, path: str) -> None:
        _check(lib().scaph_mlp_save(self._h, path.encode()))

    def load(self, path: str) -> None:
        _check(lib().scaph_mlp_load(self._h, path.encode()))


@dataclass
class BfsStats:
    levels: int
    push_levels: int
    pull_levels: int
    reached: int
    reached_edges: int
    edges_inspected: int
    alg_bytes: int
    h2d_bytes: int
    zc_bytes: int
    page_faults: int
    prefetched: int
    launches: int
    ms: float
    pcie_alg_bytes: int = 0


def _stats(s: _Stats) -> BfsStats:
    return BfsStats(s.levels, s.push_levels, s.pull_levels, s.reached, s.reached_edges, s.edges_inspected,
                    s.alg_bytes, s.h2d_bytes, s.zc_bytes, s.page_faults, s.prefetched, s.launches, s.ms,
                    s.pcie_alg_bytes)


class Engine:
    """Device BFS engine over a paged graph (scaph_engine_create)."""

    def __init__(self, graph: PagedGraph, transposed: PagedGraph | None = None, *, pool_bytes: int = 0,
                 unreached: int = UNREACHED, direction: int = DIR_ALPHABETA, alpha: float = 14.0,
                 beta: float = 96.0, block_size: int = 256, ctas_per_sm: int = 0, copy_streams: int = 2,
                 prefetch: int = 0, compact_threshold: int = 3, use_graph: int = 0, device: int = 0,
                 stream: int | None = None, record_features: int = 0, dual_timing: int = 0,
                 link_gbs: float = 0.0, giant_edges: int = 0, pull_gather_ratio: int = 0,
                 ms_compact_l2_div: int = 0, ms_compact_min_deg: int = 0, push_defer_edges: int = 0,
                 pull_warp: int = 0, pull_records: int = 0, pull_rows: int = 0, push_sparse_ratio: int = 0,
                 pull_runs: int = 0):
        self.graph, self.transposed = graph, transposed
        cfg = _Config(pool_bytes, unreached, direction, alpha, beta, block_size, ctas_per_sm, copy_streams,
                      prefetch, compact_threshold, use_graph, device, stream, record_features, dual_timing,
                      link_gbs, giant_edges, pull_gather_ratio, ms_compact_l2_div, ms_compact_min_deg, pull_warp,
                      push_defer_edges, pull_records, pull_rows, push_sparse_ratio, pull_runs)
        self._cfg = cfg
        h = C.c_void_p()
        _check(lib().scaph_engine_create(graph._h, transposed._h if transposed else None, C.byref(cfg), C.byref(h)))
        self._h = h
        self.V = graph.V

    def close(self):
        if getattr(self, "_h", None):
            lib().scaph_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bfs(self, src: int, parents: bool = False, depth_out: np.ndarray | None = None,
            parent_out: np.ndarray | None = None):
        """Runs one BFS; returns (depth, parent or None, BfsStats) as host arrays."""
        d = depth_out if depth_out is not None else np.empty(self.V, np.uint32)
        p = parent_out if parent_out is not None else (np.empty(self.V, np.uint32) if parents else None)
        st = _Stats()
        _check(lib().scaph_bfs(self._h, src, _ptr(d), _ptr(p), 0, C.byref(st)))
        return d, p, _stats(st)

    def bfs_device(self, src: int, depth_ptr: int, parent_ptr: int | None = None) -> BfsStats:
        """Runs one BFS writing into device buffers (raw CUDA pointers)."""
        st = _Stats()
        _check(lib().scaph_bfs(self._h, src, C.c_void_p(depth_ptr), C.c_void_p(parent_ptr) if parent_ptr else None,
                               1, C.byref(st)))
        return _stats(st)

    def bfs_enqueue(self, src: int, host_depth: np.ndarray) -> None:
        """Pipelined traversal with host output (scaph_bfs_enqueue): returns
        at once; host_depth (uint32[V], page-locked for overlap) is filled by
        the time sync() returns."""
        if host_depth.dtype != np.uint32 or host_depth.size < self.V or not host_depth.flags.c_contiguous:
            raise ScaphError(EINVAL, "host_depth must be a contiguous uint32 array of V entries")
        _check(lib().scaph_bfs_enqueue(self._h, src, _ptr(host_depth)))

    def bfs_async(self, src: int, depth_ptr: int, parent_ptr: int | None = None) -> None:
        """Enqueues one BFS writing into device buffers; returns at once."""
        _check(lib().scaph_bfs(self._h, src, C.c_void_p(depth_ptr), C.c_void_p(parent_ptr) if parent_ptr else None,
                               1, None))

    def msbfs(self, srcs, depth_out: np.ndarray | None = None):
        """Multi-source BFS (up to 128 sources in one traversal); returns
        (depth[nsrc][V] as host array, BfsStats)."""
        srcs = np.ascontiguousarray(srcs, np.uint32)
        d = depth_out if depth_out is not None else np.empty((len(srcs), self.V), np.uint32)
        st = _Stats()
        _check(lib().scaph_msbfs(self._h, _ptr(srcs), len(srcs), _ptr(d), 0, C.byref(st)))
        return d, _stats(st)

    def msbfs_device(self, srcs, depth_ptr: int) -> BfsStats:
        srcs = np.ascontiguousarray(srcs, np.uint32)
        st = _Stats()
        _check(lib().scaph_msbfs(self._h, _ptr(srcs), len(srcs), C.c_void_p(depth_ptr), 1, C.byref(st)))
        return _stats(st)

    def msbfs_trace(self) -> list[dict]:
        buf = (_Trace * 4096)()
        n = _check(lib().scaph_msbfs_trace(self._h, buf, 4096))
        return [{f: getattr(buf[i], f) for f, _ in _Trace._fields_} for i in range(n)]

    def set_scheduler(self, mlp: "Mlp | None") -> None:
        _check(lib().scaph_engine_set_scheduler(self._h, mlp._h if mlp is not None else None))
        self._sched = mlp  # keep the network alive while the engine uses it

    def features(self) -> np.ndarray:
        """Scheduler feature rows of the last host-loop single-source run or
        of the last multi-source run (levels x dim)."""
        dim = C.c_int()
        rows = _check(lib().scaph_bfs_features(self._h, None, 0, C.byref(dim)))
        out = np.zeros((rows, dim.value), np.float32)
        if rows:
            lib().scaph_bfs_features(self._h, _ptr(out), rows, C.byref(dim))
        return out

    def pull_pages(self, level: int, npages_in: int):
        """(unvisited vertices, their active words) per in-edge page at `level`."""
        cnt = np.zeros(npages_in, np.uint32)
        datas = np.zeros(npages_in, np.uint32)
        _check(lib().scaph_bfs_pull_pages(self._h, level, _ptr(cnt), _ptr(datas), npages_in))
        return cnt, datas

    TUNABLES = ("alpha", "beta", "block_size", "ctas_per_sm", "giant_edges", "pull_gather_ratio",
                "ms_compact_l2_div", "ms_compact_min_deg", "push_defer_edges", "pull_warp", "pull_records",
                "pull_rows", "push_sparse_ratio", "pull_runs")

    def tune(self, **kw) -> None:
        """Sets run-time tunables (scaph_engine_tune); others keep their value."""
        for k, v in kw.items():
            if k not in self.TUNABLES:
                raise ScaphError(EINVAL, f"not a tunable: {k}")
            setattr(self._cfg, k, v)
        _check(lib().scaph_engine_tune(self._h, C.byref(self._cfg)))

    _TUNABLE_DEFAULTS = {"giant_edges": 1024, "pull_gather_ratio": 64, "ms_compact_l2_div": 3,
                         "ms_compact_min_deg": 16, "push_defer_edges": 1 << 20, "pull_warp": 1,
                         "pull_rows": 2, "push_sparse_ratio": 16, "pull_runs": 1}

    def tunables(self) -> dict:
        """The tunables in force (0 fields shown as the defaults they mean)."""
        out = {k: getattr(self._cfg, k) for k in self.TUNABLES}
        for k, v in self._TUNABLE_DEFAULTS.items():
            out[k] = out[k] or v
        return out

    def evict_all(self) -> None:
        """Out-of-core engines: start the next traversal with a cold page pool."""
        _check(lib().scaph_engine_evict_all(self._h))

    def sync(self) -> None:
        _check(lib().scaph_engine_sync(self._h))

    def trace(self) -> list[dict]:
        buf = (_Trace * 4096)()
        n = _check(lib().scaph_bfs_trace(self._h, buf, 4096))
        return [{f: getattr(buf[i], f) for f, _ in _Trace._fields_} for i in range(n)]

    def page_hist(self, level: int):
        n = np.zeros(self.graph.npages, np.uint32)
        d = np.zeros(self.graph.npages, np.uint32)
        _check(lib().scaph_bfs_page_hist(self._h, level, _ptr(n), _ptr(d), self.graph.npages))
        return n, d


class Batch:
    """Mixed query batch (scaph_batch_*): several graphs resident side by
    side, many single-source queries per launch, one CUDA-graph launch per
    run."""

    def __init__(self, graphs: list, transposed: list | None = None, *, pagesize_words: int = 10 * 1024 * 1024,
                 unreached: int = UNREACHED, direction: int = DIR_ALPHABETA, alpha: float = 14.0, beta: float = 24.0,
                 device: int = 0, stream: int | None = None):
        self.graphs = list(graphs)
        arr = (_Csr * len(graphs))(*[g._c for g in graphs])
        tarr = (_Csr * len(graphs))(*[g._c for g in transposed]) if transposed else None
        cfg = _Config(0, unreached, direction, alpha, beta, 256, 0, 2, 0, 3, 0, device, stream, 0, 0, 0.0)
        h = C.c_void_p()
        _check(lib().scaph_batch_create(C.cast(arr, C.c_void_p), len(graphs),
                                        C.cast(tarr, C.c_void_p) if tarr is not None else None, pagesize_words,
                                        C.byref(cfg), C.byref(h)))
        self._h = h
        self.sizes = [int(g.V) for g in graphs]

    def close(self):
        if getattr(self, "_h", None):
            lib().scaph_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def graph_range(self, g: int) -> tuple[int, int]:
        a, n = C.c_uint32(), C.c_uint32()
        _check(lib().scaph_batch_graph_range(self._h, g, C.byref(a), C.byref(n)))
        return a.value, n.value

    @property
    def params(self) -> dict:
        p = _BatchParams()
        _check(lib().scaph_batch_get_params(self._h, C.byref(p)))
        return {"block_size": p.block_size, "ctas_per_sm": p.ctas_per_sm, "alpha": p.alpha, "beta": p.beta}

    def set_params(self, block_size: int, ctas_per_sm: int, alpha: float, beta: float) -> None:
        p = _BatchParams(block_size, ctas_per_sm, alpha, beta, 0)
        _check(lib().scaph_batch_set_params(self._h, C.byref(p)))

    def _queries(self, queries):
        q = np.ascontiguousarray(np.asarray(queries, np.uint32).reshape(-1, 2))
        if len(q) and int(q[:, 0].max()) >= len(self.sizes):
            raise ScaphError(EINVAL, f"query graph {int(q[:, 0].max())} out of range ({len(self.sizes)} graphs)")
        return q, sum(self.sizes[int(g)] for g in q[:, 0])

    def run(self, queries) -> tuple[list, BfsStats]:
        """queries: (graph, source) pairs.  Returns (one depth array per
        query, over its graph's vertices; BfsStats)."""
        q, total = self._queries(queries)
        out = np.empty(total, np.uint32)
        st = _Stats()
        _check(lib().scaph_batch_run(self._h, _ptr(q), len(q), _ptr(out), 0, C.byref(st)))
        rows, off = [], 0
        for g in q[:, 0]:
            n = self.sizes[int(g)]
            rows.append(out[off:off + n])
            off += n
        return rows, _stats(st)

    def run_device(self, queries, depth_ptr: int) -> BfsStats:
        """Depth rows into device memory at depth_ptr (u32, concatenated in
        query order)."""
        q, _ = self._queries(queries)
        st = _Stats()
        _check(lib().scaph_batch_run(self._h, _ptr(q), len(q), C.c_void_p(depth_ptr), 1, C.byref(st)))
        return _stats(st)

    def out_words(self, queries) -> int:
        return self._queries(queries)[1]

    def trace(self) -> list[dict]:
        buf = (_Trace * 4096)()
        n = _check(lib().scaph_batch_trace(self._h, buf, 4096))
        return [{f: getattr(buf[i], f) for f, _ in _Trace._fields_} for i in range(min(n, 4096))]
