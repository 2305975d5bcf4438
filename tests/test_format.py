"""Paged-CSR format and generators (host code, no GPU)."""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _digests(prefix_dir, stem="g"):
    out = {}
    for f in sorted(os.listdir(prefix_dir)):
        if f.startswith(stem + "page") or f == stem + "graph.info":
            out[f[len(stem):]] = hashlib.sha256(open(os.path.join(prefix_dir, f), "rb").read()).hexdigest()
    return out


@pytest.mark.parametrize("name", ["rmat12", "rmat17"])
def test_writer_byte_identical_to_pagegencsr_golden(tmp_path, name):
    """scaph_pages_write output == the digests of tools/pagegencsr.cpp's files."""
    meta = json.load(open(os.path.join(GOLD, "pagegencsr_digests.json")))[name]
    csr = S.Csr.rmat(meta["scale"], 16, seed=meta["seed"])
    csr.write_pages(str(tmp_path / "g"), meta["pagesize_words"])
    assert _digests(tmp_path) == meta["files"]


@pytest.mark.skipif(not os.path.exists(O.REF_PAGEGEN), reason="oracle/_ref/pagegencsr not built")
@pytest.mark.parametrize("scale,ef,seed", [(16, 16, 1), (17, 4, 2), (13, 32, 3)])
def test_writer_byte_identical_to_pagegencsr_live(tmp_path, scale, ef, seed):
    csr = S.Csr.rmat(scale, ef, seed=seed)
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    csr.write(str(b / "g"))
    subprocess.run([O.REF_PAGEGEN, str(b / "g"), "1", "u"], check=True, capture_output=True)
    csr.write_pages(str(a / "g"), 1 << 20)
    da, db = _digests(a), _digests(b)
    assert da == db and len(da) >= 3


def test_weighted_writer_byte_identical_to_pagegencsr_golden(tmp_path):
    """{ngr, wgh} pages: scaph_pages_write(weighted) == the digests of the
    files tools/pagegencsr.cpp writes with its `w` flag."""
    import tests.golden.make_weighted_pages_golden as mk

    meta = json.load(open(os.path.join(GOLD, "pagegencsr_weighted_digests.json")))
    csr = mk.graph()
    assert (csr.V, csr.E) == (meta["V"], meta["E"])
    csr.write_pages(str(tmp_path / "g"), meta["pagesize_mb"] << 20, weighted=True)
    assert _digests(tmp_path) == meta["files"]


@pytest.mark.skipif(not os.path.exists(O.REF_PAGEGEN), reason="oracle/_ref/pagegencsr not built")
@pytest.mark.parametrize("scale,ef,seed", [(14, 8, 1), (12, 32, 2), (16, 16, 3)])
def test_weighted_writer_byte_identical_to_pagegencsr_live(tmp_path, scale, ef, seed):
    c = S.Csr.rmat(scale, ef, seed=seed)
    w = np.random.default_rng(seed).integers(1, 1 << 20, c.E).astype(np.uint32)
    csr = S.Csr.from_arrays(c.idx, c.ngh, w)
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    csr.write(str(b / "g"))
    subprocess.run([O.REF_PAGEGEN, str(b / "g"), "1", "w"], check=True, capture_output=True)
    csr.write_pages(str(a / "g"), 1 << 20, weighted=True)
    da, db = _digests(a), _digests(b)
    assert da == db and len(da) >= 3


@pytest.mark.skipif(not os.path.exists(O.REF_PAGEGEN), reason="oracle/_ref/pagegencsr not built")
@pytest.mark.parametrize("weighted", [False, True])
def test_reader_opens_reference_written_pages(tmp_path, weighted):
    """scaph_graph_open on the files tools/pagegencsr.cpp itself wrote reads
    back the CSR they came from (degrees, adjacency, weights)."""
    c = S.Csr.rmat(17, 16, seed=G.SEED + 152)  # ~2M edges: several 1 Mi-word pages
    if weighted:
        w = np.random.default_rng(153).integers(1, 1000, c.E).astype(np.uint32)
        c = S.Csr.from_arrays(c.idx, c.ngh, w)
    p = str(tmp_path / "g")
    c.write(p)
    subprocess.run([O.REF_PAGEGEN, p, "1", "w" if weighted else "u"], check=True, capture_output=True)
    g = S.PagedGraph.open(p, weighted=weighted)
    assert (g.V, g.E) == (c.V, c.E) and g.npages >= 2
    assert np.array_equal(g.degree(), c.degree())
    back = g.to_csr()
    assert np.array_equal(back.idx, c.idx) and np.array_equal(back.ngh, c.ngh)
    if weighted:
        assert np.array_equal(back.wgh, c.wgh)


def test_open_roundtrip_and_degrees(tmp_path):
    csr = S.Csr.rmat(13, 16, seed=G.SEED + 60)
    p = str(tmp_path / "g")
    csr.write(p)
    csr.write_pages(p, 1 << 12)
    g = S.PagedGraph.open(p)
    assert (g.V, g.E, g.pagesize) == (csr.V, csr.E, 1 << 12)
    assert np.array_equal(g.degree(), csr.degree())
    pl = g.page_list()
    assert pl[0, 0] == 0 and pl[-1, 1] == csr.V - 1
    assert (pl[1:, 0] == pl[:-1, 1] + 1).all()
    # every page respects the cut rule 3*n + e < pagesize and is maximal
    idx = csr.idx.astype(np.int64)
    for left, right, n, e in pl:
        assert 3 * n + e < g.pagesize
        if right + 1 < csr.V:
            assert 3 * (n + 1) + idx[right + 2] - idx[left] >= g.pagesize
    back = S.Csr.read(p)
    assert np.array_equal(back.idx, csr.idx) and np.array_equal(back.ngh, csr.ngh)
    mem = S.PagedGraph.from_csr(csr, 1 << 12)
    for i in range(g.npages):
        assert np.array_equal(g.page(i), mem.page(i))


def test_corrupt_pages_rejected(tmp_path):
    csr = S.Csr.rmat(10, 16, seed=G.SEED + 61)
    p = str(tmp_path / "g")
    csr.write_pages(p, 1 << 12)
    raw = np.fromfile(p + "page0", np.uint32)
    raw[3 * 5 + 2] += 1  # node 5's degree no longer matches the edge layout
    raw.tofile(p + "page0")
    with pytest.raises(S.ScaphError) as ei:
        S.PagedGraph.open(p)
    assert ei.value.code == S.EFORMAT
    os.truncate(p + "page0", 100)
    with pytest.raises(S.ScaphError) as ei:
        S.PagedGraph.open(p)
    assert ei.value.code == S.EIO
    with pytest.raises(S.ScaphError):
        S.PagedGraph.open(str(tmp_path / "missing"))


def test_giant_vertex_rejected():
    """pagegencsr's bisection cannot place a vertex larger than a page
    (tools/pagegencsr.cpp:106-163); the writer reports it instead."""
    csr = G.star(3000, center=10)
    with pytest.raises(S.ScaphError) as ei:
        S.PagedGraph.from_csr(csr, pagesize_words=2048)
    assert ei.value.code == S.EUNSUPPORTED


def test_last_page_ending_exactly_at_V():
    """left + pagesize == V: the reference's clamp misses this case
    (tools/pagegencsr.cpp:206-207); the cut here stays inside [0, V)."""
    V = 64
    csr = G.csr_from_edges(V, np.arange(V - 1), np.arange(1, V), symmetric=False)  # out-degree 1 (last: 0)
    g = S.PagedGraph.from_csr(csr, pagesize_words=V)
    pl = g.page_list()
    assert pl[-1, 1] == V - 1 and int(pl[:, 2].sum()) == V


@pytest.mark.parametrize("gen", ["rmat", "powerlaw", "web"])
def test_generators_well_formed(gen):
    if gen == "rmat":
        c = S.Csr.rmat(12, 16, seed=5)
    elif gen == "powerlaw":
        c = S.Csr.powerlaw(5000, 60000, 1.9, 1000, seed=5)
    else:
        c = S.Csr.web(5000, 60000, 2.1, 1000, 256, 0.9, seed=5)
    idx, ngh = c.idx, c.ngh
    assert idx[0] == 0 and idx[-1] == c.E and (np.diff(idx.astype(np.int64)) >= 0).all()
    src = np.repeat(np.arange(c.V), np.diff(idx).astype(np.int64))
    assert (ngh < c.V).all() and (ngh != src).all()  # no self loops
    key = src.astype(np.int64) * c.V + ngh
    assert (np.diff(key) > 0).all()  # sorted, no duplicates
    if gen == "rmat":  # symmetric
        rev = np.sort(ngh.astype(np.int64) * c.V + src)
        assert np.array_equal(rev, key)
    if gen == "web":  # ~90 % inside the 256-id block
        local = (ngh // 256) == (src // 256)
        assert 0.8 < local.mean() < 0.97
    if gen == "powerlaw":
        assert abs(c.E - 60000) / 60000 < 0.15


def test_generators_independent_of_thread_count():
    code = ("import sys,hashlib; sys.path.insert(0,%r); import scaph_b200 as S; "
            "c=S.Csr.rmat(13,16,seed=9); p=S.Csr.powerlaw(3000,30000,1.9,500,seed=9); "
            "print(hashlib.sha256(c.ngh.tobytes()+c.idx.tobytes()+p.ngh.tobytes()).hexdigest())"
            % os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    outs = set()
    for nt in ("1", "3", "8"):
        env = dict(os.environ, OMP_NUM_THREADS=nt)
        outs.add(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                check=True).stdout.strip())
    assert len(outs) == 1


def test_transpose():
    c = S.Csr.powerlaw(3000, 30000, 1.9, 300, seed=11)
    t = c.transpose()
    src = np.repeat(np.arange(c.V), np.diff(c.idx).astype(np.int64))
    tsrc = np.repeat(np.arange(t.V), np.diff(t.idx).astype(np.int64))
    a = np.sort(src.astype(np.int64) * c.V + c.ngh)
    b = np.sort(t.ngh.astype(np.int64) * c.V + tsrc)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("scale,ef,seed,pagesize", [(12, 16, 4, 1 << 12), (15, 8, 5, 1 << 16), (16, 16, 7, 1 << 20)])
def test_streaming_writer_byte_identical(tmp_path, weighted, scale, ef, seed, pagesize):
    """scaph_pages_write_stream (edges read from the flat files a page at a
    time) writes the same bytes as scaph_pages_write, itself pinned to
    tools/pagegencsr.cpp above; and, where it was built, the same bytes as
    the reference generator run on the same flat files."""
    csr = S.Csr.rmat(scale, ef, seed=seed)
    if weighted:
        rng = np.random.default_rng(seed)
        csr = S.Csr.from_arrays(csr.idx, csr.ngh, rng.integers(1, 100, csr.E).astype(np.uint32))
    a, b, c = tmp_path / "a", tmp_path / "b", tmp_path / "c"
    for d in (a, b, c):
        d.mkdir()
    csr.write(str(c / "g"))
    assert S.pages_write_stream(str(c / "g"), str(a / "g"), pagesize, weighted) == pagesize
    csr.write_pages(str(b / "g"), pagesize, weighted=weighted)
    da = _digests(a)
    assert da == _digests(b) and len(da) >= 3
    if os.path.exists(O.REF_PAGEGEN) and pagesize == 1 << 20:
        subprocess.run([O.REF_PAGEGEN, str(c / "g"), "1", "w" if weighted else "u"], check=True, capture_output=True)
        assert da == _digests(c)


def test_streaming_writer_grows_the_page_for_a_giant_vertex(tmp_path):
    """A list longer than the page: rejected without growth, with growth the
    page becomes the smallest multiple of 4 words that holds it; the pages
    read back to the same CSR."""
    csr = G.star(3000, center=10)  # the centre has 2999 edges
    csr.write(str(tmp_path / "g"))
    with pytest.raises(S.ScaphError) as ei:
        S.pages_write_stream(str(tmp_path / "g"), str(tmp_path / "p"), 2048)
    assert ei.value.code == S.EUNSUPPORTED
    ps = S.pages_write_stream(str(tmp_path / "g"), str(tmp_path / "p"), 2048, grow=True)
    assert ps == (3 + 2999 + 1 + 3) // 4 * 4 and ps % 4 == 0
    g = S.PagedGraph.open(str(tmp_path / "p"))
    back = g.to_csr()
    assert np.array_equal(back.idx, csr.idx) and np.array_equal(back.ngh, csr.ngh)
    assert np.array_equal(g.degree(), csr.degree())


def test_streaming_writer_rejects_bad_files(tmp_path):
    csr = S.Csr.rmat(10, 8, seed=6)
    csr.write(str(tmp_path / "g"))
    ngh = np.fromfile(str(tmp_path / "g_csr.ngh"), np.uint32)
    ngh[5] = 1 << 20  # neighbour out of range
    ngh.tofile(str(tmp_path / "g_csr.ngh"))
    with pytest.raises(S.ScaphError) as ei:
        S.pages_write_stream(str(tmp_path / "g"), str(tmp_path / "p"), 1 << 12)
    assert ei.value.code == S.EFORMAT
    with pytest.raises(S.ScaphError) as ei:
        S.pages_write_stream(str(tmp_path / "missing"), str(tmp_path / "p"), 1 << 12)
    assert ei.value.code == S.EIO
