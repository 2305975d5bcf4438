"""Generates tests/golden/export_digests.json: SHA-256 digests of the text
files that the reference's own converters tools/bin2ligra.cpp,
tools/bin2ligraweight.cpp and tools/bin2totem.cpp (compiled from their
sources into oracle/_ref/ by `make -C oracle`) write for small seeded graphs,
so that the export test pins scaph_csr_export where the reference tree is
absent.  tools/bin2totemweight.cpp is not run (it reads E weights into a
buffer of V+1 words); its format is pinned against the oracle's restatement.

    python tests/golden/make_export_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import scaph_b200 as S  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import graphs as G  # noqa: E402

OUT = {"bin2ligra": ".ligra", "bin2ligraweight": ".ligra.weight", "bin2totem": ".totem"}


def graphs():
    """(name, csr with weights): a symmetric RMAT and a directed power law."""
    rng = np.random.default_rng(G.SEED + 130)
    a = S.Csr.rmat(10, 8, seed=G.SEED + 131)
    b = S.Csr.powerlaw(3000, 20000, 1.9, 500, seed=G.SEED + 132)
    out = []
    for name, c in (("rmat10", a), ("powerlaw3k", b)):
        w = rng.integers(1, 1000, c.E).astype(np.uint32)
        out.append((name, S.Csr.from_arrays(c.idx, c.ngh, w)))
    return out


def main():
    for tool in OUT:
        if not os.path.exists(O.REF_EXPORTERS[tool]):
            sys.exit(f"{O.REF_EXPORTERS[tool]} missing: run `make -C oracle` where the reference tree is present")
    digests = {}
    for name, csr in graphs():
        with tempfile.TemporaryDirectory() as tmp:
            prefix = os.path.join(tmp, "g")
            csr.write(prefix)
            files = {}
            for tool, suffix in OUT.items():
                r = subprocess.run([O.REF_EXPORTERS[tool], prefix], capture_output=True)
                if r.returncode != 0:
                    sys.exit(f"{tool} failed on {name}")
                data = open(prefix + suffix, "rb").read()
                files[suffix] = {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data)}
        digests[name] = {"V": csr.V, "E": csr.E, "files": files}
        print(f"{name}: V={csr.V} E={csr.E} {sorted(files)}")
    with open(os.path.join(HERE, "export_digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
