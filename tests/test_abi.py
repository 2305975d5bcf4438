"""The C-ABI library loads without a GPU and exports every function that
include/scaph/*.h declares; host-only entry points work on the CPU."""
import ctypes as C
import glob
import os
import re

import pytest

import scaph_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "scaph", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(scaph_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("scaph_bfs", "scaph_engine_create", "scaph_graph_open", "scaph_pages_write",
                 "scaph_bfs_page_noalloc", "scaph_last_error"):
        assert must in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = C.CDLL(S.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared but not exported"


def test_library_reports_version_and_errors():
    L = S.lib()
    assert b"sm_100a" in L.scaph_version()
    with pytest.raises(S.ScaphError) as ei:
        S.Csr.rmat(0, 16)
    assert ei.value.code == S.EINVAL and "rmat" in str(ei.value)


def test_engine_without_gpu_fails_cleanly():
    if S.device_count() > 0:
        pytest.skip("a GPU is present")
    g = S.PagedGraph.from_csr(S.Csr.rmat(8, 8, seed=1), 4096)
    with pytest.raises(S.ScaphError) as ei:
        S.Engine(g)
    assert ei.value.code == S.ECUDA


def test_fault_injection_sites():
    """The host-side fault injector knows its sites and rejects others."""
    S.fault_inject("page_copy", 0, 0)
    S.fault_inject(None)
    with pytest.raises(S.ScaphError) as ex:
        S.fault_inject("no_such_site")
    assert ex.value.code == S.EINVAL
    # an armed pinned allocation fails with ENOMEM (here there is no GPU
    # either, so the call fails whether armed or not)
    S.fault_inject("pinned_alloc", 0, 1)
    assert S.lib().scaph_host_alloc(4096) is None
    assert b"cudaMallocHost" in S.lib().scaph_last_error()
    S.fault_inject(None)
