"""Many graphs in one persistent launch (gcg_batch_pagerank) through the C ABI:
each graph's ranks against the oracle (FP32 iteration at fixed sweeps, FP64 fixed
point at the tolerance) and against its own single-graph solve, and the bounded
grid-barrier wait (failure detection without a GPU fault)."""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu


SPECS = [("rmat", 12, 1), ("er", 3000, 2), ("rmat", 9, 3), ("empty", 0, 0), ("er", 20000, 4),
         ("rmat", 14, 5), ("er", 700, 6)]


def edges(kind, n, seed):
    if kind == "rmat":
        return O.rmat_numpy(n, 16 << n, seed=seed)
    if kind == "er":
        return O.er_numpy(n, 8 * n, seed=seed)
    return np.zeros(0, np.uint32), np.zeros(0, np.uint32)


def make_graphs():
    return [gcgpu.Graph.from_edges(*edges(*sp), dedup=True) for sp in SPECS]


def nl1(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).sum() / np.abs(b).sum()


def test_batch_against_oracle():
    gs = make_graphs()
    oracles = [O.OracleGraph(*edges(*sp)) for sp in SPECS]
    with gcgpu.Batch(gs) as b:
        r, sw, res, st = b.pagerank(max_sweeps=20, tol=0.0)
        for g, go, part in zip(gs, oracles, b.split(r)):
            assert g.num_vertices == go.nv and g.num_edges == go.ne
            ref, n, _ = go.pagerank_jacobi(max_sweeps=20)
            assert nl1(part, ref) <= 1e-6
        r, sw, res, st = b.pagerank(max_sweeps=1000, tol=1e-8)
        assert st.converged == 1
        for k, (go, part) in enumerate(zip(oracles, b.split(r))):
            f64, _ = go.pagerank_jacobi_f64(max_sweeps=3000, tol=1e-12)
            assert nl1(part, f64) <= 1e-6, k
            o32, n32, _ = go.pagerank_jacobi(max_sweeps=1000, tol=1e-8)
            # near 1e-8 the FP32 residual is a few ulps per vertex and depends on the
            # summation order, so on small graphs the stopping sweep can differ more
            assert nl1(part, o32) <= 1e-6 and abs(int(sw[k]) - n32) <= max(8, n32 // 4), (k, sw[k], n32)
    for g in gs:
        g.free()


def test_batch_fixed_sweeps_equal_single_graph_solves():
    gs = make_graphs()
    with gcgpu.Batch(gs) as b:
        r, sw, res, st = b.pagerank(max_sweeps=20, tol=0.0)
        assert list(sw) == [20] * len(gs)
        for g, part in zip(gs, b.split(r)):
            ref, _ = g.pagerank(max_sweeps=20)
            assert np.array_equal(part, ref)
    for g in gs:
        g.free()


def test_batch_to_tolerance_matches_single_graph_solves():
    gs = make_graphs()
    with gcgpu.Batch(gs) as b:
        r, sw, res, st = b.pagerank(max_sweeps=1000, tol=1e-8)
        assert st.converged == 1 and np.all(res <= 1e-8)
        for k, (g, part) in enumerate(zip(gs, b.split(r))):
            ref, rst = g.pagerank(max_sweeps=1000, tol=1e-8)
            assert abs(int(sw[k]) - rst.sweeps) <= 1, (k, sw[k], rst.sweeps)
            if int(sw[k]) == rst.sweeps:
                assert np.array_equal(part, ref)
            else:
                assert np.abs(part - ref).sum() / np.abs(ref).sum() <= 1e-6
        # uneven sizes converge at different sweeps, all in one persistent launch:
        # init (3), the persistent kernel, the scatter, the layout map to the output
        assert st.kernel_launches == 6
        # warm start from the answer: every graph stops within two sweeps
        r2, sw2, res2, st2 = b.pagerank(max_sweeps=1000, tol=1e-8, init_rank=r)
        assert np.all(sw2 <= 2) and np.all(res2 <= 1e-8)
        assert st2.kernel_launches == 7
    for g in gs:
        g.free()


def test_batch_barrier_timeout_is_reported_and_context_survives():
    gs = make_graphs()[:3]
    with gcgpu.Batch(gs) as b:
        with pytest.raises(gcgpu.GcgError) as e:
            b.pagerank(max_sweeps=5, flags=gcgpu.PR_TEST_BARRIER_TIMEOUT)
        assert e.value.status == -7
        r, sw, res, st = b.pagerank(max_sweeps=5)
        assert list(sw) == [5, 5, 5]
        ref, _ = gs[0].pagerank(max_sweeps=5)
        assert np.array_equal(b.split(r)[0], ref)
    for g in gs:
        g.free()


def test_batch_graph_replay_and_launch_configs_keep_results():
    gs = make_graphs()
    with gcgpu.Batch(gs) as b:
        r1, sw1, res1, st1 = b.pagerank(max_sweeps=1000, tol=1e-8)
        assert b.config()[2]  # the solve was captured into a CUDA graph
        r2, sw2, res2, _ = b.pagerank(max_sweeps=1000, tol=1e-8)  # replayed
        assert np.array_equal(r1, r2) and np.array_equal(sw1, sw2) and np.array_equal(res1, res2)
        # every launch configuration computes the same sums in the same order
        for hub, run in [(0, 0), (8192, 1), (100000, 4), (16384, 16)]:
            b.set_config(hub, run)
            r3, sw3, res3, _ = b.pagerank(max_sweeps=1000, tol=1e-8)
            assert np.array_equal(r1, r3) and np.array_equal(sw1, sw3) and np.array_equal(res1, res3), (hub, run)
        hub, run, ms = b.autotune(sweeps=4)
        assert ms > 0 and run in (0, 1, 4, 16)
        h2, q2, ready = b.config()
        assert (h2, q2) == (hub, run) and not ready
        r4, sw4, _, _ = b.pagerank(max_sweeps=1000, tol=1e-8)
        assert np.array_equal(r1, r4) and np.array_equal(sw1, sw4)
    for g in gs:
        g.free()


def test_batch_one_hub_layout_against_oracle():
    """GCG_BATCH_ONE_HUB: one hub over the union's hottest sources and the union's
    rows in id order (the layout the batch falls back to when its ids are too wide
    for per-graph relabelling). Chunk boundaries differ from the single-graph
    plans, so each graph is checked against the oracle: the FP32 iteration at
    fixed sweeps and the FP64 fixed point at the tolerance; every launch
    configuration of this layout gives the same bits."""
    gs = make_graphs()
    oracles = [O.OracleGraph(*edges(*sp)) for sp in SPECS]
    with gcgpu.Batch(gs, one_hub=True) as b:
        r, sw, res, st = b.pagerank(max_sweeps=20, tol=0.0)
        assert list(sw) == [20] * len(gs)
        for g, go, part in zip(gs, oracles, b.split(r)):
            assert g.num_vertices == go.nv and g.num_edges == go.ne
            ref, n, _ = go.pagerank_jacobi(max_sweeps=20)
            assert nl1(part, ref) <= 1e-6
        r1, sw1, res1, st = b.pagerank(max_sweeps=1000, tol=1e-8)
        assert st.converged == 1
        for k, (go, part) in enumerate(zip(oracles, b.split(r1))):
            f64, _ = go.pagerank_jacobi_f64(max_sweeps=3000, tol=1e-12)
            assert nl1(part, f64) <= 1e-6, k
        for hub, run in [(0, 0), (8192, 1), (100000, 4), (16384, 16)]:
            b.set_config(hub, run)
            r3, sw3, res3, _ = b.pagerank(max_sweeps=1000, tol=1e-8)
            assert np.array_equal(r1, r3) and np.array_equal(sw1, sw3) and np.array_equal(res1, res3), (hub, run)
    for g in gs:
        g.free()
