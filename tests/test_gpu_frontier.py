"""Selective scheduling on the device frontier (the reference's bitset_scheduler),
through the C ABI: CC by label propagation with and without the scheduler against
the oracle's labels, delta PageRank against plain Jacobi, and the per-sweep
progress log (the reference's .deltalog fields)."""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheduler", [False, True])
@pytest.mark.parametrize("sym", [True, False])
def test_label_propagation_fixpoint_vs_oracle(scheduler, sym):
    s, d = O.rmat_numpy(13, 4 << 13, seed=41)  # sparse enough for many components
    go = O.OracleGraph(s, d, symmetrise=sym)
    ref, _ = go.cc()
    log = np.zeros(1000, np.int32)
    with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=sym) as g:
        lab, st = g.connected_components(algorithm=gcgpu.CC_LABEL_PROPAGATION, scheduler=scheduler,
                                         frontier_log=log)
        uf, ust = g.connected_components()
    assert np.array_equal(lab, ref) and np.array_equal(uf, ref)
    assert st.ncomponents == ust.ncomponents and st.passes >= 2
    f = log[:st.passes]
    if scheduler:
        # iteration 0 updates everything, the frontier then shrinks to nothing
        assert f[0] == go.nv and f[-1] < f[0] and np.all(f > 0)
    else:
        assert np.all(f == go.nv)


def test_label_propagation_needs_whole_neighbourhoods():
    s, d = O.er_numpy(1000, 3000, seed=2)
    with gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=False) as g:
        with pytest.raises(gcgpu.GcgError) as e:
            g.connected_components(algorithm=gcgpu.CC_LABEL_PROPAGATION)
        assert e.value.status == -6


def test_delta_pagerank_threshold_zero_equals_jacobi():
    s, d = O.rmat_numpy(12, 16 << 12, seed=43)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        ref, _ = g.pagerank(max_sweeps=15)
        r, st = g.pagerank(mode=gcgpu.PR_DELTA, max_sweeps=15, delta_threshold=0.0)
        assert st.sweeps == 15
        l1 = np.abs(r.astype(np.float64) - ref).sum() / np.abs(ref).sum()
        assert l1 <= 1e-6


def test_delta_pagerank_schedules_less_and_stays_close():
    s, d = O.rmat_numpy(14, 16 << 14, seed=44)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        n, E = g.num_vertices, g.num_edges
        ref, rst = g.pagerank(max_sweeps=1000, tol=1e-10)
        wl = np.zeros(2 * 1000, np.uint64)
        dl = np.zeros(1000, np.float64)
        r, st = g.pagerank(mode=gcgpu.PR_DELTA, max_sweeps=1000, delta_threshold=1e-4, work_log=wl, delta_log=dl)
        k = st.sweeps
        assert st.converged == 1 and k > 2
        upd = wl[0:2 * k:2]
        work = wl[1:2 * k:2]
        assert upd[0] == n and np.all(np.diff(upd.astype(np.int64)) > 0) and np.all(np.diff(work.astype(np.int64)) >= 0)
        # after sweep 0 only vertices with a scheduled in-neighbour run (the ones
        # without in-edges never again), and the run ends by an empty frontier
        per = np.diff(np.concatenate([[0], upd.astype(np.int64)]))
        nz = int((g.degrees()[:, 0] > 0).sum())
        assert np.all(per[1:] <= nz) and upd[-1] < n * k
        assert np.all(dl[:k] >= 0)
        l1 = np.abs(r.astype(np.float64) - ref).sum() / np.abs(ref).sum()
        assert l1 <= 1e-3, l1


def test_jacobi_delta_and_work_logs():
    s, d = O.rmat_numpy(12, 16 << 12, seed=45)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        n, E = g.num_vertices, g.num_edges
        res = np.zeros(10, np.float64)
        dl = np.zeros(10, np.float64)
        wl = np.zeros(20, np.uint64)
        r, st = g.pagerank(max_sweeps=10, residuals=res, delta_log=dl, work_log=wl)
        r9, _ = g.pagerank(max_sweeps=9)
        # the last sweep's sum |r' - r| and its normalised form
        d9 = np.abs(r.astype(np.float64) - r9.astype(np.float64)).sum()
        assert abs(dl[9] - d9) <= 1e-6 * d9 + 1e-12
        assert abs(res[9] - dl[9] / np.abs(r.astype(np.float64)).sum()) <= 1e-9
        assert list(wl[0::2]) == [n * (i + 1) for i in range(10)]
        assert list(wl[1::2]) == [E * (i + 1) for i in range(10)]
