"""The allocation-free PageRank entry point (gcg_pagerank_csr_noalloc).

It serves callers that cannot let a library call cudaMalloc/cudaFree: a host
framework whose own allocator owns the GPU's memory, or a loop that must not
take the synchronisation a device allocation or free can cause. They hand over
a CSR, out-degrees and an output vector already in their device memory; the
library's only scratch is a fixed static device array.

Checked here through the C ABI: two calls in a row agree with the regular
entry point (gcg_pagerank on a graph built by the device sharder) and with the
oracle's FP64 Jacobi iteration within the PageRank tolerance used everywhere
else (normalised L1 <= 1e-6); each sweep that ran logs its residual and the
slots after the last one stay untouched; sizes beyond the scratch limit and
host arrays are rejected. This file is collected last so that a run stopping
at the first failure has run every other test.
"""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu
L1_TOL = 1e-6


def nl1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / np.abs(b).sum()


def _device_csr(scale, seed):
    import torch
    s, d = O.rmat_numpy(scale, 16 << scale, seed=seed)
    g = gcgpu.Graph.from_edges(s, d, dedup=True)
    rp, col = g.csr(gcgpu.CSR_IN)
    od = g.degrees()[:, 1].astype(np.uint32)
    dev = lambda a: torch.from_numpy(a.view(np.int32)).cuda()  # noqa: E731
    return g, dev(rp), dev(col), dev(od), O.OracleGraph(s, d)


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    g, rp, col, od, go = _device_csr(16, 5)
    n = g.num_vertices
    assert n <= gcgpu.NOALLOC_MAX_VERTICES and n == go.nv
    for kw in (dict(max_sweeps=3), dict(max_sweeps=300, tol=1e-8)):
        ref, rst = g.pagerank(**kw)
        f64, _ = go.pagerank_jacobi_f64(max_sweeps=kw["max_sweeps"], tol=kw.get("tol", 0.0))
        for _ in range(2):  # the scratch keeps the previous call's contents
            out = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
            res = torch.full((kw["max_sweeps"],), -7.0, dtype=torch.float64, device="cuda")
            st = gcgpu.pagerank_csr_noalloc(rp, col, od, out, residuals=res, **kw)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert nl1(got, ref) <= L1_TOL
            assert nl1(got, f64) <= L1_TOL
            log = res.cpu().numpy()
            assert np.all(log[:st.sweeps] >= 0.0) and np.all(log[st.sweeps:] == -7.0)
            assert log[st.sweeps - 1] == st.residual and st.device_ms > 0.0
            if kw.get("tol"):
                assert st.converged == 1 and st.residual <= kw["tol"]
                assert abs(st.sweeps - rst.sweeps) <= max(3, rst.sweeps // 10)
            else:
                assert st.sweeps == 3
    g.free()


def test_noalloc_rejects_oversize_and_host_arrays():
    import torch
    g, rp, col, od, _ = _device_csr(10, 6)
    out = torch.zeros(g.num_vertices, dtype=torch.float32, device="cuda")
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.pagerank_csr_noalloc(rp, col, od, out, num_vertices=gcgpu.NOALLOC_MAX_VERTICES + 1)
    assert e.value.status == -6 and "scratch limit" in str(e.value)
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.pagerank_csr_noalloc(rp, col, od, np.zeros(g.num_vertices, np.float32))
    assert e.value.status == -1 and "device memory" in str(e.value)
    g.free()
