"""The ctypes mirrors in scaph_b200 against the C structs of
include/scaph/scaph.h: a small C program compiled against the header prints
sizeof and offsetof of every field, and each must equal the ctypes layout
(a field added to the header but not to the mirror, or in another order,
would shift every later field the library reads).  CPU only."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import pytest

import scaph_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (C struct, its ctypes mirror); the mirrors use the header's field names,
# padding fields included
MIRRORS = [
    ("scaph_csr", S._Csr),
    ("scaph_graph_info", S._GraphInfo),
    ("scaph_config", S._Config),
    ("scaph_bfs_stats", S._Stats),
    ("scaph_query", S._Query),
    ("scaph_batch_params", S._BatchParams),
    ("scaph_level_trace", S._Trace),
]


@pytest.fixture(scope="module")
def c_layout():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "scaph/scaph.h"', "int main(void) {"]
    for name, mirror in MIRRORS:
        lines.append(f'    printf("%s size %zu\\n", "{name}", sizeof({name}));')
        for f, _ in mirror._fields_:
            lines.append(f'    printf("%s %s %zu %zu\\n", "{name}", "{f}", offsetof({name}, {f}), '
                         f'sizeof((({name} *)0)->{f}));')
    lines += ["    return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        r = subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    sizes, fields = {}, {}
    for line in out.splitlines():
        p = line.split()
        if p[1] == "size":
            sizes[p[0]] = int(p[2])
        else:
            fields[(p[0], p[1])] = (int(p[2]), int(p[3]))
    return sizes, fields


@pytest.mark.parametrize("name,mirror", MIRRORS, ids=[m[0] for m in MIRRORS])
def test_ctypes_mirror_matches_header(c_layout, name, mirror):
    sizes, fields = c_layout
    assert C.sizeof(mirror) == sizes[name], f"{name}: ctypes {C.sizeof(mirror)} B, C {sizes[name]} B"
    for f, t in mirror._fields_:
        off, size = fields[(name, f)]
        assert getattr(mirror, f).offset == off, f"{name}.{f}: ctypes offset {getattr(mirror, f).offset}, C {off}"
        assert C.sizeof(t) == size, f"{name}.{f}: ctypes size {C.sizeof(t)}, C {size}"
