"""scaph_bfs_page_noalloc: the BFS entry point that allocates no device memory.

It exists for callers that must not have the library call cudaMalloc (hosts
that keep all GPU memory in their own pool, latency-critical paths where
cudaMalloc/cudaFree would synchronise the device).  Its scratch state is a
fixed __device__ array shared by every call.  This test calls it through the
C ABI twice in a row on the same device page and checks each result against
the regular entry point (scaph_bfs through an engine): depths bit-exact,
parents a valid BFS tree.  The second call starts from the first call's
leftovers in the shared array, so it also checks that each call clears what
it needs.  The file is named to be collected last.
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
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_scaph_bfs_twice():
    import torch

    csr = S.Csr.rmat(14, 16, seed=G.SEED + 40)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 21)
    assert g.npages == 1
    left, right, n, e = (int(x) for x in g.page_list()[0])
    assert left == 0 and n == csr.V and e == csr.E
    words = (3 * n + e + 3) // 4 * 4
    d_page = torch.from_numpy(g.page(0)[:words].view(np.int32).copy()).cuda()
    eng = S.Engine(g)
    f = _entry()
    stream = torch.cuda.current_stream()
    srcs = [int(np.argmax(csr.degree()))] + G.sources(csr, 1, 40)
    for src in srcs:  # two calls in a row
        ref_depth, _, _ = eng.bfs(src)
        d_depth = torch.full((n,), 12345, dtype=torch.int32, device="cuda")
        d_parent = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        rc = f(d_page.data_ptr(), n, e, src, S.UNREACHED, d_depth.data_ptr(), d_parent.data_ptr(),
               stream.cuda_stream)
        assert rc == 0, S.lib().scaph_last_error().decode()
        torch.cuda.synchronize()
        depth = d_depth.cpu().numpy().view(np.uint32)
        parent = d_parent.cpu().numpy().view(np.uint32)
        assert np.array_equal(depth, ref_depth), f"src {src}: depths differ from scaph_bfs"
        rc, bad = O.validate_tree(csr.idx, csr.ngh, src, depth, parent)
        assert rc == 0, f"src {src}: invalid BFS tree (code {rc} at {bad})"
    eng.close()


def test_noalloc_rejects_oversize_graph():
    import torch

    f = _entry()
    d_page = torch.zeros(16, dtype=torch.int32, device="cuda")
    d_depth = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = f(d_page.data_ptr(), (1 << 18) + 1, 0, 0, S.UNREACHED,
           d_depth.data_ptr(), None, None)
    assert rc == S.EINVAL
    assert b"SCAPH_NOALLOC_MAX_V" in S.lib().scaph_last_error()
    rc = f(d_page.data_ptr(), 4, (1 << 22) + 1, 0, S.UNREACHED, d_depth.data_ptr(), None, None)
    assert rc == S.EINVAL
