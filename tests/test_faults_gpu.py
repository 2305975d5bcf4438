"""Host-side failure injection on the GPU path: a failing pinned allocation,
device allocation, host-page registration or page copy makes the C ABI
return a status (never abort), leaves nothing half-built, and the library
works again once the fault is gone.  The reference ends the process on any
CUDA error (H_ERR -> exit, src/gpu_engine.cuh:28-39).  No GPU fault is
involved: the injected calls are never made."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def disarm():
    S.fault_inject(None)
    yield
    S.fault_inject(None)


@pytest.fixture(scope="module")
def small():
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 70)
    return csr, S.PagedGraph.from_csr(csr, pagesize_words=1 << 12)


def test_pinned_allocation_failure():
    S.fault_inject("pinned_alloc", 0, 1)
    assert S.lib().scaph_host_alloc(1 << 20) is None
    assert b"cudaMallocHost" in S.lib().scaph_last_error()
    p = S.lib().scaph_host_alloc(1 << 20)  # the next one is not armed
    assert p is not None
    S.lib().scaph_host_free(p)


def test_device_allocation_failure_at_create(small):
    csr, g = small
    S.fault_inject("device_alloc", 0, 1)
    with pytest.raises(S.ScaphError) as ex:
        S.Engine(g)
    assert ex.value.code == S.ECUDA
    eng = S.Engine(g)
    src = G.sources(csr, 1, 70)[0]
    d, _, _ = eng.bfs(src)
    assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src))
    eng.close()


def test_host_register_failure_out_of_core():
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 71)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 12)  # a graph never pinned before
    S.fault_inject("host_register", 0, 1)
    with pytest.raises(S.ScaphError) as ex:
        S.Engine(g, pool_bytes=4 * g.pagesize * 4)
    assert ex.value.code == S.ECUDA
    eng = S.Engine(g, pool_bytes=4 * g.pagesize * 4)
    src = G.sources(csr, 1, 71)[0]
    d, _, _ = eng.bfs(src)
    assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src))
    eng.close()


def test_page_copy_failure_mid_traversal(small):
    """A page copy that cannot be issued in the middle of an out-of-core
    traversal: scaph_bfs returns ECUDA; the same engine then runs exactly."""
    csr, g = small
    eng = S.Engine(g, pool_bytes=4 * g.pagesize * 4, compact_threshold=0)  # copies only
    src = G.sources(csr, 1, 72)[0]
    eng.evict_all()
    S.fault_inject("page_copy", 2, 1)
    with pytest.raises(S.ScaphError) as ex:
        eng.bfs(src)
    assert ex.value.code == S.ECUDA and "copy not issued" in str(ex.value)
    S.fault_inject(None)
    eng.sync()
    for cold in (True, False):
        if cold:
            eng.evict_all()
        d, _, st = eng.bfs(src)
        assert np.array_equal(d, O.bfs(csr.idx, csr.ngh, src))
    eng.close()


def test_page_copy_failure_in_multi_source(small):
    csr, g = small
    eng = S.Engine(g, pool_bytes=4 * g.pagesize * 4, compact_threshold=0)
    srcs = G.sources(csr, 8, 73)
    eng.evict_all()
    S.fault_inject("page_copy", 1, 1)
    with pytest.raises(S.ScaphError):
        eng.msbfs(srcs)
    S.fault_inject(None)
    eng.sync()
    d, _ = eng.msbfs(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(d[i], O.bfs(csr.idx, csr.ngh, s))
    eng.close()
