"""Applications on the App-hook API, run on the GPU: the example BFS / SSSP /
WCC programs (scaph_b200/apps) against the hook oracle, graph resident and
out of core, and the reference's own applications built unchanged against
the compat headers (when they were built)."""
import os
import re
import subprocess

import numpy as np
import pytest

import scaph_b200 as S
from oracle import oracle as O
from tests import graphs as G
from tests.test_apps import FAR_BFS, FAR_SSSP, single_source, weighted

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "scaph_b200", "apps", "_build")
PAGE = 1 << 12  # 16 KiB pages: the test graphs span dozens of pages


@pytest.fixture(scope="module")
def graphs(tmp_path_factory):
    d = tmp_path_factory.mktemp("apps")
    sym = S.Csr.rmat(13, 8, seed=G.SEED + 90)
    dire = S.Csr.powerlaw(20000, 200000, 1.9, 2000, seed=G.SEED + 91)
    wdir = weighted(dire, 92)
    out = {}
    for name, csr, w in (("sym", sym, False), ("dir", dire, False), ("wdir", wdir, True)):
        prefix = str(d / name)
        csr.write_pages(prefix, PAGE, weighted=w)
        out[name] = (prefix, csr)
    return out


def run_app(app, prefix, out, *args, ref=False):
    exe = os.path.join(BUILD, "ref", app) if ref else os.path.join(BUILD, app)
    if not os.access(exe, os.X_OK):
        pytest.skip(f"{exe} not built")
    cmd = [exe, f"--graphfile={prefix}"] + ([f"--out={out}"] if out else []) + list(args)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (cmd, r.stdout[-2000:], r.stderr[-2000:])
    info = {}
    m = re.search(r"path=(\w+) rounds=(\d+) seconds=\S+ h2d=(\d+) zc=(\d+) faults=(\d+) pool_pages=(\d+) pages=(\d+)",
                  r.stdout)
    if m:
        info = dict(path=m.group(1), rounds=int(m.group(2)), h2d=int(m.group(3)), zc=int(m.group(4)),
                    faults=int(m.group(5)), pool_pages=int(m.group(6)), pages=int(m.group(7)))
    values = np.fromfile(out, np.uint32) if out else None
    return values, info, r.stdout


@pytest.mark.parametrize("name,far", [("sym", FAR_BFS), ("sym", 0xFFFFFFFF), ("dir", 0xFFFFFFFF), ("dir", 4)])
def test_bfs_app_single_source_runs_the_bfs_engine(graphs, tmp_path, name, far):
    prefix, csr = graphs[name]
    for src in G.sources(csr, 2, 93):
        got, info, _ = run_app("bfs", prefix, tmp_path / "v", f"--src={src}", f"--far={far}")
        assert info["path"] == "engine"
        assert np.array_equal(got, np.minimum(O.bfs(csr.idx, csr.ngh, src, unreached=far), far))


def test_bfs_app_two_sources_runs_the_hooks(graphs, tmp_path):
    prefix, csr = graphs["dir"]
    a, b = G.sources(csr, 2, 94)
    got, info, _ = run_app("bfs", prefix, tmp_path / "v", f"--sources={a},{b}")
    assert info["path"] == "hooks" and info["rounds"] > 1
    value = np.full(csr.V, FAR_BFS, np.uint32)
    value[[a, b]] = 0
    active = np.zeros(csr.V, np.uint8)
    active[[a, b]] = 1
    assert np.array_equal(got, O.hook_fixpoint(csr.idx, csr.ngh, "bfs", value, active))


def test_sssp_app(graphs, tmp_path):
    prefix, csr = graphs["wdir"]
    for src in G.sources(csr, 2, 95):
        got, info, _ = run_app("sssp", prefix, tmp_path / "v", f"--src={src}")
        assert info["path"] == "hooks"
        value, active = single_source(csr.V, src, FAR_SSSP)
        assert np.array_equal(got, O.hook_fixpoint(csr.idx, csr.ngh, "sssp", value, active, wgh=csr.wgh))
        assert np.array_equal(got, O.sssp_dijkstra(csr.idx, csr.ngh, csr.wgh, src, FAR_SSSP))


@pytest.mark.parametrize("name", ["sym", "dir"])
def test_wcc_app(graphs, tmp_path, name):
    prefix, csr = graphs[name]
    got, info, _ = run_app("wcc", prefix, tmp_path / "v")
    assert info["path"] == "hooks"
    assert np.array_equal(got, O.min_reaching_id(csr.idx, csr.ngh))


@pytest.mark.parametrize("app,name", [("bfs", "dir"), ("sssp", "wdir"), ("wcc", "dir")])
def test_apps_out_of_core(graphs, tmp_path, app, name):
    """--max_memory=1 MiB leaves room for a fraction of the pages: the page
    store (hooks) or the BFS engine's pager streams the rest."""
    prefix, csr = graphs[name]
    src = G.sources(csr, 1, 96)[0]
    got, info, _ = run_app(app, prefix, tmp_path / "v", f"--src={src}", "--max_memory=1", "--threshold=1")
    assert info["pool_pages"] < info["pages"]
    assert info["faults"] + info["zc"] > 0
    if app == "bfs":
        ref = np.minimum(O.bfs(csr.idx, csr.ngh, src, unreached=FAR_BFS), FAR_BFS)
    elif app == "sssp":
        ref = O.sssp_dijkstra(csr.idx, csr.ngh, csr.wgh, src, FAR_SSSP)
    else:
        ref = O.min_reaching_id(csr.idx, csr.ngh)
    assert np.array_equal(got, ref)


def test_reference_wcc_app_checks_itself(graphs):
    """The reference's app/wcc.cu, unmodified: its own check() (a CPU
    labelling, app/wcc.cu:59-92) compares the GPU result."""
    prefix, _ = graphs["dir"]
    _, _, out = run_app("wcc", prefix, None, "--check", ref=True)
    assert "total error count: 0" in out, out[-2000:]


def test_reference_bfs_and_sssp_apps_run(graphs):
    prefix, csr = graphs["sym"]
    src = G.sources(csr, 1, 97)[0]
    _, _, out = run_app("bfs", prefix, None, f"--src={src}", ref=True)
    assert out.count("scaph: run") == 11 and "BFS engine" in out  # 10 timed runs + 1 (app/bfs.cu:146-166)
    prefix, _ = graphs["wdir"]
    _, _, out = run_app("sssp", prefix, None, f"--src={src % 20000}", "--check", ref=True)
    assert "check passed!" in out


def run_pr(prefix, out, *args):
    exe = os.path.join(BUILD, "pr")
    if not os.access(exe, os.X_OK):
        pytest.skip(f"{exe} not built")
    cmd = [exe, f"--graphfile={prefix}", f"--out={out}"] + list(args)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (cmd, r.stdout[-2000:], r.stderr[-2000:])
    m = re.search(r"pagerank iters=(\d+) l1=(\S+) ms=\S+ resident=(\d) h2d=(\d+) zc=(\d+) faults=(\d+)", r.stdout)
    assert m, r.stdout
    return np.fromfile(out, np.float32), dict(iters=int(m.group(1)), l1=float(m.group(2)),
                                             resident=int(m.group(3)), h2d=int(m.group(4)), zc=int(m.group(5)))


# float32 ranks with float32 atomic sums against the float64 power iteration
PR_RTOL, PR_ATOL = 1e-4, 1e-8


@pytest.mark.parametrize("name", ["sym", "dir", "wdir"])
@pytest.mark.parametrize("memory", [None, "1"], ids=["resident", "out-of-core"])
def test_pagerank_app(graphs, tmp_path, name, memory):
    """PageRank on the page store (§8(f)1: the reference's app/pr.cu does not
    build): resident and out of core, symmetric, directed and weighted pages,
    within PR_RTOL of the float64 oracle."""
    prefix, csr = graphs[name]
    args = ["--iters=25"] + (["--weighted"] if name == "wdir" else [])
    if memory:
        args += [f"--max_memory={memory}", "--threshold=1"]
    got, info = run_pr(prefix, tmp_path / "r", *args)
    ref = O.pagerank(csr.idx, csr.ngh, 25, 0.85)
    assert got.shape == ref.shape
    assert np.allclose(got, ref, rtol=PR_RTOL, atol=PR_ATOL), float(np.max(np.abs(got - ref) / ref))
    assert abs(float(got.astype(np.float64).sum()) - 1.0) < 1e-3
    page_bytes = S.PagedGraph.open(prefix, weighted=name == "wdir").npages * PAGE * 4
    out_of_core = memory is not None and page_bytes > int(memory) << 20
    assert info["resident"] == (0 if out_of_core else 1)
    if out_of_core:
        assert info["h2d"] + info["zc"] > 0
