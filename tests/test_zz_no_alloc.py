"""scaph_bfs_page_noalloc: the BFS entry point that allocates no device memory.

It exists for callers that must not have the library call cudaMalloc (hosts
that keep all GPU memory in their own pool, latency-critical paths where
cudaMalloc/cudaFree would synchronise the device).  Its scratch state is a
fixed __device__ array shared by every call.  These tests call it through the
C ABI and check each result against the CPU oracle (depths bit-exact, parents
a valid BFS tree) and against the regular entry point (scaph_bfs through an
engine), two calls in a row: the second call starts from the first call's
leftovers in the shared array, so it also checks that each call clears what
it needs.  They also cover directed pages (push only), a path deeper than
the engine's 4096-level graph loop, a page with a corrupt Node record, and
oversize inputs.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu


def _entry():
    f = S.lib().scaph_bfs_page_noalloc
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_page(csr, pagesize_words=1 << 21):
    """The graph as one device-resident page (the layout of <p>page0)."""
    import torch

    g = S.PagedGraph.from_csr(csr, pagesize_words=pagesize_words)
    assert g.npages == 1
    left, right, n, e = (int(x) for x in g.page_list()[0])
    assert left == 0 and n == csr.V and e == csr.E
    words = (3 * n + e + 3) // 4 * 4
    return g, torch.from_numpy(g.page(0)[:words].view(np.int32).copy()).cuda(), n, e


def _run(f, d_page, n, e, src, flags, unreached=S.UNREACHED):
    import torch

    stats = S._Stats()
    d_depth = torch.full((n,), 12345, dtype=torch.int32, device="cuda")
    d_parent = torch.full((n,), 7, dtype=torch.int32, device="cuda")
    rc = f(d_page.data_ptr(), n, e, src, unreached, flags, d_depth.data_ptr(), d_parent.data_ptr(),
           C.addressof(stats), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, S.lib().scaph_last_error().decode()
    torch.cuda.synchronize()
    return d_depth.cpu().numpy().view(np.uint32), d_parent.cpu().numpy().view(np.uint32), stats


def test_noalloc_matches_oracle_and_scaph_bfs_twice():
    csr = S.Csr.rmat(14, 16, seed=G.SEED + 40)
    g, d_page, n, e = _device_page(csr)
    eng = S.Engine(g)
    f = _entry()
    srcs = [int(np.argmax(csr.degree()))] + G.sources(csr, 1, 40)
    pulls = 0
    for src in srcs:  # two calls in a row
        depth, parent, st = _run(f, d_page, n, e, src, S.NOALLOC_SYMMETRIC)
        assert np.array_equal(depth, O.bfs(csr.idx, csr.ngh, src)), f"src {src}: depths differ from the oracle"
        ref_depth, _, _ = eng.bfs(src)
        assert np.array_equal(depth, ref_depth), f"src {src}: depths differ from scaph_bfs"
        rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
        assert rc == 0, f"src {src}: invalid BFS tree (code {rc} at {bad})"
        assert st.levels == st.push_levels + st.pull_levels
        pulls += st.pull_levels
    # alpha/beta switches to pull on this RMAT graph: the pull kernel ran
    assert pulls > 0
    eng.close()


def test_noalloc_directed_page_pushes_only():
    """A directed page: without SCAPH_NOALLOC_SYMMETRIC every level pushes,
    and the depths equal the oracle's."""
    csr = S.Csr.powerlaw(20000, 200000, zipf_s=1.9, max_degree=2000, seed=G.SEED + 41)
    assert not csr.symmetric()
    _, d_page, n, e = _device_page(csr)
    f = _entry()
    for src in G.sources(csr, 2, 41):
        depth, parent, st = _run(f, d_page, n, e, src, 0)
        assert np.array_equal(depth, O.bfs(csr.idx, csr.ngh, src))
        assert st.pull_levels == 0 and st.levels > 1
        rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
        assert rc == 0, f"invalid BFS tree (code {rc} at {bad})"


def test_noalloc_deep_path():
    """A 5000-vertex path: 5000 levels, every depth exact (no level cap)."""
    csr = G.path(5000)
    _, d_page, n, e = _device_page(csr)
    f = _entry()
    depth, _, st = _run(f, d_page, n, e, 0, S.NOALLOC_SYMMETRIC)
    assert st.levels == 5000
    assert np.array_equal(depth, np.arange(5000, dtype=np.uint32))
    depth, _, _ = _run(f, d_page, n, e, 2500, S.NOALLOC_SYMMETRIC)
    assert np.array_equal(depth, O.bfs(csr.idx, csr.ngh, 2500))


def test_noalloc_rejects_corrupt_node_record():
    """A correctly sized page whose Node record points past the edges."""
    import torch

    csr = G.random_graph(3000, 12000, seed=42)
    _, d_page, n, e = _device_page(csr)
    v = int(np.flatnonzero(csr.degree() > 0)[17])
    bad = d_page.clone()
    bad[3 * v + 1] = e  # Node{vtx, idx, len} of v: idx + len > edgenum
    f = _entry()
    d_depth = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = f(bad.data_ptr(), n, e, 0, S.UNREACHED, S.NOALLOC_SYMMETRIC, d_depth.data_ptr(), None, None, None)
    assert rc == S.EFORMAT
    # the untouched page still runs afterwards
    depth, _, _ = _run(f, d_page, n, e, 5, S.NOALLOC_SYMMETRIC)
    assert np.array_equal(depth, O.bfs(csr.idx, csr.ngh, 5))


def test_noalloc_rejects_bad_arguments():
    import torch

    f = _entry()
    d_page = torch.zeros(16, dtype=torch.int32, device="cuda")
    d_depth = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = f(d_page.data_ptr(), (1 << 18) + 1, 0, 0, S.UNREACHED, 0, d_depth.data_ptr(), None, None, None)
    assert rc == S.EINVAL
    assert b"SCAPH_NOALLOC_MAX_V" in S.lib().scaph_last_error()
    rc = f(d_page.data_ptr(), 4, (1 << 22) + 1, 0, S.UNREACHED, 0, d_depth.data_ptr(), None, None, None)
    assert rc == S.EINVAL
    # the engine rejects a sentinel below 2; so does this entry point
    rc = f(d_page.data_ptr(), 4, 0, 0, 1, 0, d_depth.data_ptr(), None, None, None)
    assert rc == S.EINVAL
    rc = f(d_page.data_ptr(), 4, 0, 0, S.UNREACHED, 0x10, d_depth.data_ptr(), None, None, None)
    assert rc == S.EINVAL
