"""A graph past 2^31 edges (R-MAT scale 27, 2.28 G raw edges, ~2.2 G after dedup,
about 80 GB of device memory at the peak): the device sharder and one PageRank
sweep, checked through properties that do not depend on the size. Degree sums
equal the edge count, row pointers end at it, and after one sweep from 1.0 the
rank mass is 0.15 V + 0.85 x (vertices with out-edges), since every such vertex
hands out exactly its rank."""
import numpy as np
import pytest

import gcgpu

pytestmark = pytest.mark.gpu


def test_sharder_and_sweep_beyond_2_pow_31_edges():
    import torch

    scale, m = 27, 17 << 27
    free, _ = torch.cuda.mem_get_info()
    if free < 110 << 30:
        pytest.skip("needs ~110 GB of free device memory")
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty(m, dtype=torch.int32, device="cuda")
    gcgpu.generate_rmat(scale, m, 0.57, 0.19, 0.19, seed=27, src=s, dst=d)
    with gcgpu.Graph.from_edges(s, d, dedup=True, nshards=64, out_csr=False) as g:
        del s, d
        V, E = g.num_vertices, g.num_edges
        assert (1 << scale) - (1 << 16) < V <= 1 << scale and (1 << 31) < E <= m  # V = max id + 1
        deg = g.degrees()
        assert int(deg[:, 0].astype(np.int64).sum()) == E
        assert int(deg[:, 1].astype(np.int64).sum()) == E
        iv = g.intervals()
        assert iv[-1] == V - 1 and np.all(np.diff(iv.astype(np.int64)) > 0)
        r = torch.empty(V, dtype=torch.float32, device="cuda")
        _, st = g.pagerank(max_sweeps=1, init=1.0, out=r)
        assert st.sweeps == 1
        mass = float(r.double().sum())
        with_out = int((deg[:, 1] > 0).sum())
        want = 0.15 * V + 0.85 * with_out
        assert abs(mass - want) <= 1e-5 * want, (mass, want)
    torch.cuda.empty_cache()
    gcgpu.release_cached_memory()
