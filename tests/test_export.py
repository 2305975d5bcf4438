"""Text exports of the flat CSR (scaph_csr_export) against the reference's
converters tools/bin2ligra.cpp, bin2ligraweight.cpp, bin2totem.cpp: byte for
byte, through committed digests of their output and, where the reference tree
was present at build time, by running them (oracle/_ref).  bin2totemweight.cpp
reads E weights into a buffer of V+1 words (tools/bin2totemweight.cpp:94-96)
and is not run; that format is pinned by the oracle's restatement, which the
three converters pin in turn."""
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
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KINDS = {"ligra": S.EXPORT_LIGRA, "ligra.weight": S.EXPORT_LIGRA_WEIGHT, "totem": S.EXPORT_TOTEM,
         "weight.totem": S.EXPORT_TOTEM_WEIGHT}
TOOL = {"ligra": "bin2ligra", "ligra.weight": "bin2ligraweight", "totem": "bin2totem"}
HAVE_REF = all(os.path.exists(p) for p in O.REF_EXPORTERS.values())


def weighted(csr: S.Csr, seed: int) -> S.Csr:
    w = np.random.default_rng(seed).integers(1, 1000, csr.E).astype(np.uint32)
    return S.Csr.from_arrays(csr.idx, csr.ngh, w)


def export(csr: S.Csr, prefix: str, kind: str) -> bytes:
    csr.write(prefix)
    path = S.csr_export(prefix, KINDS[kind])
    assert path == prefix + S.EXPORT_SUFFIX[KINDS[kind]]
    return open(path, "rb").read()


def cases():
    return [("rmat11", weighted(S.Csr.rmat(11, 8, seed=G.SEED + 140), 141)),
            ("powerlaw", weighted(S.Csr.powerlaw(5000, 30000, 1.9, 800, seed=G.SEED + 142), 143)),
            ("ragged_isolated", weighted(G.random_graph(1001, 900, seed=G.SEED + 144), 145)),
            ("single_vertex", S.Csr.from_arrays(np.zeros(2, np.uint64), np.zeros(0, np.uint32),
                                                np.zeros(0, np.uint32))),
            ("path", weighted(G.path(40), 146))]


def test_matches_reference_golden(tmp_path):
    """Same bytes as the reference converters wrote for the committed cases
    (tests/golden/make_export_golden.py made the digests)."""
    import tests.golden.make_export_golden as mk

    gold = json.load(open(os.path.join(GOLD, "export_digests.json")))
    for name, csr in mk.graphs():
        assert (csr.V, csr.E) == (gold[name]["V"], gold[name]["E"])
        for suffix, meta in gold[name]["files"].items():
            data = export(csr, str(tmp_path / name), suffix[1:])
            assert len(data) == meta["bytes"] and hashlib.sha256(data).hexdigest() == meta["sha256"], (name, suffix)


@pytest.mark.parametrize("kind", list(KINDS))
def test_matches_oracle_restatement(tmp_path, kind):
    for name, csr in cases():
        data = export(csr, str(tmp_path / name), kind)
        ref = O.export_text(csr.idx.astype(np.uint32), csr.ngh, csr.wgh, kind)
        assert data == ref, (name, kind)


@pytest.mark.skipif(not HAVE_REF, reason="reference converters not built (oracle/_ref)")
@pytest.mark.parametrize("kind", list(TOOL))
def test_matches_reference_live(tmp_path, kind):
    """Runs the reference converter on the same files; also pins the
    oracle's restatement of its format."""
    for name, csr in cases()[:3]:
        a, b = str(tmp_path / (name + "_ours")), str(tmp_path / (name + "_ref"))
        ours = export(csr, a, kind)
        csr.write(b)
        r = subprocess.run([O.REF_EXPORTERS[TOOL[kind]], b], capture_output=True)
        assert r.returncode == 0, r.stderr
        ref = open(b + "." + kind, "rb").read()
        assert ours == ref, (name, kind)
        assert O.export_text(csr.idx.astype(np.uint32), csr.ngh, csr.wgh, kind) == ref


def test_errors(tmp_path):
    with pytest.raises(S.ScaphError) as e:
        S.csr_export(str(tmp_path / "missing"), S.EXPORT_LIGRA)
    assert e.value.code == S.EIO
    csr = G.path(10)
    csr.write(str(tmp_path / "g"))
    with pytest.raises(S.ScaphError) as e:
        S.csr_export(str(tmp_path / "g"), 9)
    assert e.value.code == S.EINVAL


def test_command_line(tmp_path):
    csr = weighted(G.path(12), 147)
    prefix = str(tmp_path / "g")
    csr.write(prefix)
    r = subprocess.run([sys.executable, "-m", "scaph_b200.export", "bin2totemweight", prefix],
                       capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert open(prefix + "weight.totem", "rb").read() == \
        O.export_text(csr.idx.astype(np.uint32), csr.ngh, csr.wgh, "weight.totem")
    r = subprocess.run([sys.executable, "-m", "scaph_b200.export", "bin2nothing", prefix],
                       capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 2
