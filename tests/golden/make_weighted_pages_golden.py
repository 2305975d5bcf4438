"""Generates tests/golden/pagegencsr_weighted_digests.json: SHA-256 digests of
the weighted paged-CSR files ({ngr, wgh} edge pairs) that the reference's own
tools/pagegencsr.cpp (compiled into oracle/_ref/pagegencsr by `make -C
oracle`, run with the `w` flag) writes for a small seeded weighted graph.

    python tests/golden/make_weighted_pages_golden.py
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

CASE = {"scale": 15, "ef": 8, "seed": G.SEED + 150, "weight_seed": 151, "pagesize_mb": 1}


def graph():
    c = S.Csr.rmat(CASE["scale"], CASE["ef"], seed=CASE["seed"])
    w = np.random.default_rng(CASE["weight_seed"]).integers(1, 1 << 20, c.E).astype(np.uint32)
    return S.Csr.from_arrays(c.idx, c.ngh, w)


def main():
    if not os.path.exists(O.REF_PAGEGEN):
        sys.exit(f"{O.REF_PAGEGEN} missing: run `make -C oracle` where the reference tree is present")
    csr = graph()
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "g")
        csr.write(prefix)
        subprocess.run([O.REF_PAGEGEN, prefix, str(CASE["pagesize_mb"]), "w"], check=True, capture_output=True)
        files = {f[1:]: hashlib.sha256(open(os.path.join(tmp, f), "rb").read()).hexdigest()
                 for f in sorted(os.listdir(tmp)) if f.startswith("gpage") or f == "ggraph.info"}
    out = dict(CASE, V=csr.V, E=csr.E, files=files)
    with open(os.path.join(HERE, "pagegencsr_weighted_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"V={csr.V} E={csr.E} {sorted(files)}")


if __name__ == "__main__":
    main()
