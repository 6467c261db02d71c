"""Batched personalised PageRank (gcg_ppr_batched) through the C ABI, against the
oracle restatement (orc_ppr) and the scalar personalised path of gcg_pagerank.
Tolerance: per-source normalised L1 <= 1e-6 (rows longer than one 256-edge
segment are summed in segment order, a different float order than the oracle)."""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu
L1_TOL = 1e-6
TELE = 1.0 - 0.85  # the oracle's restart mass, (1 - damping) in double


def per_source_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return (np.abs(a - b).sum(axis=0) / np.maximum(np.abs(b).sum(axis=0), 1e-300)).max()


@pytest.mark.parametrize("scale,k,seed", [(10, 40, 1), (12, 256, 2), (11, 300, 3), (9, 1, 4)])
def test_ppr_batched_vs_oracle(scale, k, seed):
    s, d = O.rmat_numpy(scale, 16 << scale, seed=seed)
    go = O.OracleGraph(s, d)
    rng = np.random.default_rng(seed)
    src = rng.integers(0, go.nv, k).astype(np.uint32)
    ref, n = go.ppr(src, damping=0.85, max_sweeps=25, tol=0.0)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        out, st = g.ppr_batched(src, max_sweeps=25, teleport=TELE)
    assert st.sweeps == 25
    assert per_source_l1(out, ref) <= L1_TOL


def test_ppr_batched_converges_and_matches_scalar_personalised():
    s, d = O.er_numpy(5000, 60000, seed=9)
    src = np.array([0, 17, 4999, 17, 2500], np.uint32)  # a repeated source too
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        res = np.zeros(500, np.float64)
        out, st = g.ppr_batched(src, max_sweeps=500, teleport=TELE, tol=1e-8, residuals=res)
        assert st.converged == 1 and st.residual <= 1e-8
        assert np.all(np.diff(res[:20]) <= 0) or res[19] < res[0]
        for j, v in enumerate(src):
            r, sst = g.pagerank(max_sweeps=500, teleport=TELE, tol=1e-8, source=int(v))
            assert sst.converged == 1
            l1 = np.abs(r.astype(np.float64) - out[:, j]).sum() / np.abs(out[:, j]).sum()
            assert l1 <= 1e-6, (j, l1)
        assert np.array_equal(out[:, 1], out[:, 3])


def test_ppr_batched_per_source_stop_and_compaction():
    # 200 sources on a graph where many reach little (dangling or low out-reach):
    # they stop early, the matrix is compacted 256 -> 128 -> 64 -> 32 columns, and
    # every column still equals its own scalar personalised solve and the oracle
    s, d = O.rmat_numpy(12, 16 << 12, seed=21)
    go = O.OracleGraph(s, d)
    rng = np.random.default_rng(21)
    src = rng.integers(0, go.nv, 200).astype(np.uint32)
    ref, n_ref = go.ppr(src, damping=0.85, max_sweeps=300, tol=1e-8)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        out, st = g.ppr_batched(src, max_sweeps=300, teleport=TELE, tol=1e-8)
        # near 1e-8 the normalised change is at the FP32 noise floor, so sums in
        # another order cross tol a few sweeps apart (the scalar path's tests allow
        # the same)
        assert st.converged == 1 and abs(st.sweeps - n_ref) <= max(3, n_ref // 10)
        assert per_source_l1(out, ref) <= L1_TOL
        for j in rng.choice(200, 12, replace=False):
            r, sst = g.pagerank(max_sweeps=300, teleport=TELE, tol=1e-8, source=int(src[j]))
            l1 = np.abs(r.astype(np.float64) - out[:, j]).sum() / np.abs(out[:, j]).sum()
            assert l1 <= 1e-6, (j, l1)


def test_ppr_batched_device_output_and_validation():
    import torch
    s, d = O.rmat_numpy(10, 16 << 10, seed=5)
    src = np.arange(64, dtype=np.uint32) * 3
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        host, _ = g.ppr_batched(src, max_sweeps=10, teleport=TELE)
        dev = torch.zeros((g.num_vertices, 64), dtype=torch.float32, device="cuda")
        tsrc = torch.from_numpy(src.view(np.int32)).cuda()
        g.ppr_batched(tsrc, max_sweeps=10, teleport=TELE, out=dev)
        assert np.array_equal(dev.cpu().numpy(), host)
        with pytest.raises(gcgpu.GcgError):
            g.ppr_batched(np.array([g.num_vertices], np.uint32))


def test_scalar_personalised_pagerank_vs_oracle():
    s, d = O.rmat_numpy(10, 16 << 10, seed=7)
    go = O.OracleGraph(s, d)
    src = np.array([5], np.uint32)
    ref, _ = go.ppr(src, damping=0.85, max_sweeps=30, tol=0.0)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        r, st = g.pagerank(max_sweeps=30, teleport=TELE, source=5)
    assert np.abs(r - ref[:, 0]).sum() / np.abs(ref[:, 0]).sum() <= L1_TOL


def test_ppr_batched_work_log_counts_the_sources_still_iterating():
    # without a tolerance every source runs every sweep: the log grows by k x (V, E)
    s, d = O.rmat_numpy(10, 16 << 10, seed=5)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        V, E, k, S = g.num_vertices, g.num_edges, 40, 25
        src = np.random.default_rng(5).integers(0, V, k).astype(np.uint32)
        wl = np.zeros(2 * S, np.uint64)
        _, st = g.ppr_batched(src, max_sweeps=S, teleport=TELE, work_log=wl)
        i = np.arange(1, S + 1, dtype=np.uint64)
        assert np.array_equal(wl[0::2], i * k * V) and np.array_equal(wl[1::2], i * k * E)
        # with one: sources leave as they converge, so the increments shrink, the
        # first is all k sources and the log stays flat after the last sweep
        S = 300
        src = np.random.default_rng(6).integers(0, V, 64).astype(np.uint32)
        wl = np.zeros(2 * S, np.uint64)
        _, st = g.ppr_batched(src, max_sweeps=S, teleport=TELE, tol=1e-8, work_log=wl)
        upd, gat = wl[0::2].astype(np.int64), wl[1::2].astype(np.int64)
        assert np.array_equal(gat * V, upd * E)
        inc = np.diff(np.concatenate([[0], gat]))
        assert inc[0] == 64 * E and np.all(np.diff(inc) <= 0)
        assert inc[st.sweeps - 1] >= E and np.all(inc[st.sweeps:] == 0)
