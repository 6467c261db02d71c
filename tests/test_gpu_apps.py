"""The C++ drop-in apps (graphchi-cpp_b200/apps, built on the header-only shim
over the C ABI) run like the reference's example apps: same command line, same
output files. Checked against the oracle on an edge-list file."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "graphchi-cpp_b200", "bin")


def run(app, *opts):
    r = subprocess.run([os.path.join(BIN, app)] + list(opts), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture()
def edgelist(tmp_path):
    s, d = O.rmat_numpy(10, 8 << 10, seed=51)
    cs, cd = O.canonical_edges(s, d, symmetrise=False, dedup=True)
    path = str(tmp_path / "g.el")
    O.write_edgelist(path, cs, cd)
    return path, O.OracleGraph(cs, cd)


def test_pagerank_app_vertex_api_bitexact(edgelist):
    path, go = edgelist
    run("pagerank", f"file={path}", "niters=4")
    got = O.read_vout(path, np.float32)
    ref = go.pagerank_gs_inmem(4)
    assert np.array_equal(got[:go.nv], ref)


def test_pagerank_app_tolerance_and_scheduler_write_deltalog(edgelist):
    path, go = edgelist
    for extra in (["tol=1e-8"], ["scheduler=1", "niters=200", "delta_threshold=0"]):
        run("pagerank", f"file={path}", *extra)
        lines = open(path + ".deltalog").read().split()
        rows = [l.split(",") for l in lines]
        assert len(rows) > 3 and all(len(r) == 4 for r in rows)
        it = [int(r[0]) for r in rows]
        upd = [int(r[1]) for r in rows]
        assert it == list(range(len(rows))) and upd == sorted(upd) and upd[0] == go.nv
        assert all(float(r[3]) >= 0 for r in rows)


@pytest.mark.parametrize("scheduler", [0, 1])
def test_connectedcomponents_app(edgelist, scheduler):
    path, go = edgelist
    run("connectedcomponents", f"file={path}", f"scheduler={scheduler}")
    got = O.read_vout(path, np.uint32)
    ref, _ = go.cc()
    assert np.array_equal(got[:go.nv], ref)
    assert os.path.exists(path + ".components")


def test_trianglecounting_app(edgelist):
    path, go = edgelist
    total, _, _ = go.tc()
    out = run("trianglecounting", f"file={path}", f"assertequals={int(total)}")
    assert str(int(total)) in out


@pytest.mark.parametrize("mode", ["sync", "semisync"])
def test_pagerank_functional_app_runs_the_kernel_on_the_device(edgelist, mode):
    # the reference's functional kernel (gather / apply / scatter methods) compiled
    # with nvcc and run by graphchi_gpu/functional_gpu.cuh: bulk-synchronous
    # PageRank with teleport 0.15/N, as pagerank_functional --mode sync
    path, go = edgelist
    run("pagerank_functional", f"file={path}", "niters=10", f"mode={mode}")
    got = O.read_vout(path, np.float32)[:go.nv].astype(np.float64)
    ref, _, _ = go.pagerank_jacobi(teleport=0.15 / go.nv, damping=0.85, init=1.0, max_sweeps=9)
    ref = np.asarray(ref, np.float64)
    assert np.abs(got - ref).sum() / np.abs(ref).sum() <= 1e-6


def test_bulksync_smoketest_app_pins_bulk_synchronous_visibility(edgelist):
    # the reference's src/tests/bulksync_functional_test.cpp run by the device
    # functional plug-in: every gather sees the previous iteration, every scatter
    # the value just computed; three expectations per in-edge and iteration
    path, go = edgelist
    out = run("bulksync_smoketest", f"file={path}", "niters=5")
    assert "Smoketest passed successfully" in out
    checks = int([line for line in out.splitlines() if line.startswith("checks ")][0].split()[1])
    assert checks == 3 * 4 * len(go.src)
    got = O.read_vout(path, np.int32)
    assert np.all(got[:go.nv] == 4)


@pytest.mark.parametrize("case", ["handmade_components", "rmat_s12_ef8_sym_seed2"])
def test_connectedcomponents_app_components_file_matches_reference(tmp_path, case):
    # the whole drop-in path (edge list -> device CC -> .vout -> analyze_labels)
    # against the .components file the reference's own app wrote for the same input
    import json
    g = np.load(os.path.join(ROOT, "tests", "golden", f"{case}.npz"))
    spec = json.loads(str(g["spec"]))
    if spec["kind"] == "explicit":
        s, d = np.array(spec["src"], np.uint32), np.array(spec["dst"], np.uint32)
    else:
        s, d = O.rmat_numpy(spec["scale"], spec["ef"] << spec["scale"], seed=spec["seed"])
    cs, cd = O.canonical_edges(s, d, symmetrise=spec.get("sym", False), dedup=True)
    path = str(tmp_path / "g.el")
    O.write_edgelist(path, cs, cd)
    out = run("connectedcomponents", f"file={path}")
    assert np.array_equal(O.read_vout(path, np.uint32)[: int(g["nv"])], g["cc"])
    assert open(path + ".components", "rb").read() == bytes(g["cc_components"])
    assert "Total number of different labels" in out


def test_pagerank_app_edge_program_matches_reference_files(tmp_path):
    # with num_vertices * 4 >= membudget the app runs the edge-value program
    # (pagerank.cpp:166-177), as the reference app did on this input: the .vout bit
    # for bit and the .deltalog as the engine wrote it (counts exact, each delta
    # to its printed 6 decimals)
    import hashlib
    import json
    g = np.load(os.path.join(ROOT, "tests", "golden", "er_n300000_m2400000_seed7.npz"))
    spec = json.loads(str(g["spec"]))
    s, d = O.er_numpy(spec["n"], spec["m"], spec["seed"])
    cs, cd = O.canonical_edges(s, d, symmetrise=False, dedup=True)
    path = str(tmp_path / "g.el")
    O.write_edgelist(path, cs, cd)
    out = run("pagerank", f"file={path}", "niters=5", "nshards=4", "membudget_mb=1")
    assert "in-memory mode" not in out
    vals = O.read_vout(path, np.float32)[: int(g["nv"])]
    assert hashlib.sha256(vals.tobytes()).hexdigest() == str(g["pr_edge_5_4_1_sha"])
    got = [ln.split(",") for ln in open(path + ".deltalog").read().split()]
    ref = [ln.split(",") for ln in bytes(g["pr_edge_5_4_1_deltalog"]).decode().split()]
    assert [r[:3] for r in got] == [r[:3] for r in ref]
    np.testing.assert_allclose([float(r[3]) for r in got], [float(r[3]) for r in ref], rtol=0, atol=2e-6)


@pytest.mark.parametrize("tag", ["pr_gs_4_1_0", "pr_gs_4_4_1", "pr_gs_6_2_0"])
def test_pagerank_app_in_memory_program_matches_reference_files(tmp_path, tag):
    # the in-memory program as the reference app ran it (niters, nshards, membudget
    # from the tag): the .vout bit for bit and the .deltalog byte for byte (one line
    # when the engine ran in its single-shard in-memory mode, one per iteration else)
    g = np.load(os.path.join(ROOT, "tests", "golden", "rmat_s10_ef16_seed1.npz"))
    s, d = O.rmat_numpy(10, 16 << 10, seed=1)
    cs, cd = O.canonical_edges(s, d, symmetrise=False, dedup=True)
    path = str(tmp_path / "g.el")
    O.write_edgelist(path, cs, cd)
    niters, P, budget = (int(x) for x in tag.split("_")[2:])
    opts = [f"file={path}", f"niters={niters}", f"nshards={P}"] + ([f"membudget_mb={budget}"] if budget else [])
    out = run("pagerank", *opts)
    assert "in-memory mode" in out
    assert np.array_equal(O.read_vout(path, np.float32)[: int(g["nv"])], g[tag])
    assert open(path + ".deltalog", "rb").read() == bytes(g[tag + "_deltalog"])
