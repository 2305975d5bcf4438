#!/usr/bin/env python3
"""Generates the golden fixtures in tests/golden/ (run where the reference
tree is available, i.e. where oracle/_ref was built from it).

For each small seeded graph and source it stores the CPU oracle's depths in
both conventions (sentinel 63 as in app/bfs.cu:18, and 0xFFFFFFFF), but only
after the REFERENCE's own bfs::check (app/bfs.cu:67-117, compiled from source
into oracle/_ref/libscaphref.so) has reported "total errors: 0" for them.

It also stores SHA-256 digests of the paged-CSR files that the reference's
own tools/pagegencsr.cpp (compiled into oracle/_ref/pagegencsr) writes for
two graphs, so that the writer can be checked without the reference, and
golden outputs of the reference's compress_stat and chunk-mask helpers.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import scaph_b200 as S  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import graphs as G  # noqa: E402

UNR = 0xFFFFFFFF


def graphs():
    yield "rmat10", S.Csr.rmat(10, 16, seed=G.SEED + 100)
    yield "rmat12", S.Csr.rmat(12, 8, seed=G.SEED + 101)
    yield "path100", G.path(100)
    yield "star600", G.star(600, center=3)
    yield "ragged1001", G.random_graph(1001, 1500, seed=102)
    yield "powerlaw4k", S.Csr.powerlaw(4000, 40000, 1.9, 500, seed=G.SEED + 103)


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/libscaphref.so missing: build it with `make -C oracle` next to the reference tree")
    out = {}
    for name, csr in graphs():
        idx, ngh = csr.idx.copy(), csr.ngh.copy()
        srcs = sorted(set([int(np.argmax(csr.degree()))] + G.sources(csr, 3, 104)))
        if name == "path100":
            srcs = [0, 50]
        d63, dnat = [], []
        for s in srcs:
            a = O.bfs(idx, ngh, s, 63)
            b = O.bfs(idx, ngh, s, UNR)
            err, _ = O.ref_bfs_check(idx.astype(np.uint32), ngh, s, a)
            if err != 0:
                sys.exit(f"{name} src {s}: reference bfs::check reports {err} mismatches")
            d63.append(a)
            dnat.append(b)
        np.savez_compressed(os.path.join(HERE, f"bfs_{name}.npz"), idx=idx, ngh=ngh,
                            sources=np.array(srcs, np.uint32), depth63=np.stack(d63), depth=np.stack(dnat))
        print(f"{name}: V={csr.V} E={csr.E} sources={srcs} (reference check: 0 errors)")

    # paged-CSR files written by the reference generator
    digests = {}
    for name, csr, mwords in [("rmat12", S.Csr.rmat(12, 16, seed=G.SEED + 110), 1),
                              ("rmat17", S.Csr.rmat(17, 16, seed=G.SEED + 111), 1)]:
        with tempfile.TemporaryDirectory() as tmp:
            p = os.path.join(tmp, "g")
            csr.write(p)
            r = subprocess.run([O.REF_PAGEGEN, p, str(mwords), "u"], capture_output=True, text=True)
            if r.returncode != 0:
                sys.exit(f"pagegencsr failed on {name}")
            files = sorted(f for f in os.listdir(tmp) if f.startswith("gpage") or f == "ggraph.info")
            digests[name] = {"seed": G.SEED + (110 if name == "rmat12" else 111),
                             "scale": 12 if name == "rmat12" else 17, "pagesize_words": mwords << 20,
                             "files": {f[1:]: hashlib.sha256(open(os.path.join(tmp, f), "rb").read()).hexdigest()
                                       for f in files}}
        print(f"pagegencsr {name}: {len(digests[name]['files'])} files")
    with open(os.path.join(HERE, "pagegencsr_digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)

    # compress_stat (src/compress.h:18-40) on one page with a seeded stat
    csr = S.Csr.rmat(11, 16, seed=G.SEED + 120)
    g = S.PagedGraph.from_csr(csr, pagesize_words=1 << 13)
    rng = np.random.default_rng(121)
    pl = g.page_list()
    comp = {}
    for p in range(min(g.npages, 3)):
        left, right, n, e = (int(x) for x in pl[p])
        stat = (rng.random(csr.V) < 0.2).astype(np.uint8)
        src = g.page(p).copy()
        dst = np.zeros(g.pagesize, np.uint32)
        active = int(stat[left:right + 1].sum())
        cnt = O.rlib().ref_compress_stat(O._p(src), O._p(dst), O._p(stat), left, n, active)
        comp[f"page{p}"] = {"active": int(cnt), "stat_seed": 121, "sha256": hashlib.sha256(dst.tobytes()).hexdigest()}
        np.save(os.path.join(HERE, f"compress_stat_page{p}.npy"), stat)
    # chunk-mask helpers (src/tools.h:11-85)
    rng = np.random.default_rng(122)
    masks = [0, 0xFFFFFFFF, 0x80000001, 0x0F0F0F0F] + [int(x) for x in rng.integers(0, 2**32, 60, dtype=np.uint64)]
    chunks = []
    for m in masks:
        sm = m - (1 << 32) if m >= (1 << 31) else m
        row = {"mask": m, "max": O.rlib().ref_max_zero_run(sm),
               "fit": [O.rlib().ref_fit_zero_run(sm, r) for r in range(1, 33)]}
        chunks.append(row)
    with open(os.path.join(HERE, "chunk_and_compress.json"), "w") as f:
        json.dump({"compress_stat": {"graph": {"scale": 11, "seed": G.SEED + 120, "pagesize_words": 1 << 13},
                                     "pages": comp}, "chunk_masks": chunks}, f, indent=1)
    print("compress_stat + chunk masks: done")


if __name__ == "__main__":
    main()
