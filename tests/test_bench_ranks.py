"""The multi-process path of bench.py on the CPU (gloo, world size 2; the engine
runs one replica per GPU, with no collective on the data path): the job's time is
the slowest rank's, its GTEPS count every replica's edges, and the reference arm
runs on rank 0 only while the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        ms = bench.max_over_ranks(10.0 + rank, world, "cpu")  # rank 1 is the slower replica
        gteps = bench.whole_job_gteps(2.0e9, world, ms / 1e3)
        q.put((rank, ms, gteps))
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank_and_rate_counts_all_replicas():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, gteps in got:
        assert ms == 11.0
        assert gteps == pytest.approx(2.0e9 * 2 / 0.011 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.whole_job_gteps(1.0e9, 1, 0.5) == pytest.approx(2.0)


def test_reference_arm_under_torchrun_runs_on_rank_zero_only():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "pagerank")):
        pytest.skip("oracle/_ref is not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "2", "--warmup", "1", "--scale", "12"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "reference"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["e2e"]["d2h_bytes_per_step"] == 0
    # the same workload as the GPU arm (scale 12 here), one step = one timed iteration
    assert rec["config"]["workload"] == "pagerank_rmat12_ef16_to_1e-08"
    assert len(rec["cpu_baseline"]["iteration_s"]) == 2 and rec["ms_per_step"] > 0
    # the value is the engine's in-memory mode (one shard, large budget); the default
    # configuration's run is reported beside it
    assert "in-memory mode" in rec["cpu_baseline"]["sample"]
    db = rec["cpu_baseline"]["default_budget"]
    assert db["value"] > 0 and len(db["iteration_s"]) == 2, db


def test_reference_arm_loads_no_library_code():
    # the reference arm makes its input with the oracle's generator restatement:
    # nothing of the library under test runs on the reference's path
    src = open(os.path.join(ROOT, "bench.py")).read()
    body = src[src.index("def reference_iterations("):src.index("def oracle_check(")]
    assert "gcgpu" not in body
