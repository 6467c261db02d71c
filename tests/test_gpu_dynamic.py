"""Dynamic graphs through the C ABI (gcg_graph_add_edges / gcg_graph_delete_edges,
the batched counterpart of graphchi_dynamicgraph_engine's edge insertion and
deletion): after each batch the resident graph equals the oracle's graph of the
resulting edge list (CSRs, degrees, intervals bit-exact) and a graph built from
scratch on it, and algorithms on it give the oracle's answers."""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu


def same_graph(a, b):
    ia, ib = a.info(), b.info()
    assert (ia.num_vertices, ia.num_edges, ia.nshards, ia.has_out_csr) == \
        (ib.num_vertices, ib.num_edges, ib.nshards, ib.has_out_csr)
    for which in ([gcgpu.CSR_IN, gcgpu.CSR_OUT] if ia.has_out_csr else [gcgpu.CSR_IN]):
        ra, ca = a.csr(which)
        rb, cb = b.csr(which)
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
    assert np.array_equal(a.degrees(), b.degrees())
    assert np.array_equal(a.intervals(), b.intervals())


def same_as_oracle(g, s, d, sym, nshards):
    go = O.OracleGraph(s, d, symmetrise=sym, nv=g.num_vertices)
    assert g.num_edges == go.ne
    rp, col = g.csr(gcgpu.CSR_IN)
    assert np.array_equal(rp, go.in_rowptr) and np.array_equal(col, go.in_col)
    if g.info().has_out_csr:
        rp, col = g.csr(gcgpu.CSR_OUT)
        assert np.array_equal(rp, go.out_rowptr) and np.array_equal(col, go.out_col)
    assert np.array_equal(g.degrees(), go.degrees())
    assert np.array_equal(g.intervals(), go.intervals(nshards))
    return go


def remove_pairs(s, d, ds, dd):
    keys = (s.astype(np.uint64) << 32) | d
    gone = (ds.astype(np.uint64) << 32) | dd
    keep = ~np.isin(keys, gone)
    return s[keep], d[keep]


@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("device_input", [False, True])
def test_add_then_delete_equals_fresh_build(sym, device_input):
    s, d = O.rmat_numpy(11, 8 << 11, seed=61)
    a_s, a_d = O.er_numpy(2500, 3000, seed=62)  # ids beyond the R-MAT graph's: the vertex count grows
    rng = np.random.default_rng(63)
    pick = rng.choice(len(s), 700, replace=False)
    del_s = np.concatenate([s[pick], a_s[:100], np.array([5000], np.uint32)])  # one absent edge too
    del_d = np.concatenate([d[pick], a_d[:100], np.array([7], np.uint32)])
    conv = (lambda x: x)
    if device_input:
        import torch
        conv = (lambda x: torch.from_numpy(x.astype(np.int32)).cuda())
    with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=sym, nshards=8) as g:
        g.pagerank(mode=gcgpu.PR_GS_EXACT, max_sweeps=2)  # builds the level schedule of the old edges
        g.add_edges(conv(a_s), conv(a_d))
        s2, d2 = np.concatenate([s, a_s]), np.concatenate([d, a_d])
        with gcgpu.Graph.from_edges(s2, d2, dedup=True, symmetrise=sym, nshards=8) as ref:
            same_graph(g, ref)
            assert g.num_vertices == max(int(s2.max()), int(d2.max())) + 1
        same_as_oracle(g, s2, d2, sym, 8)
        g.delete_edges(conv(del_s), conv(del_d))
        if sym:  # an undirected edge goes in both directions
            del_s, del_d = np.concatenate([del_s, del_d]), np.concatenate([del_d, del_s])
        s3, d3 = remove_pairs(s2, d2, del_s, del_d)
        if sym:
            # the symmetrised build adds the reverse of every kept pair: drop pairs whose reverse is deleted
            s3, d3 = remove_pairs(s3, d3, del_d, del_s)
        with gcgpu.Graph.from_edges(s3, d3, dedup=True, symmetrise=sym, nshards=8,
                                    num_vertices=g.num_vertices) as ref:
            same_graph(g, ref)
            # plans built before the updates are rebuilt: answers equal the fresh graph's
            r1, _ = g.pagerank(max_sweeps=10)
            r2, _ = ref.pagerank(max_sweeps=10)
            assert np.array_equal(r1, r2)
            l1, _ = g.connected_components()
            l2, _ = ref.connected_components()
            assert np.array_equal(l1, l2)
        go = same_as_oracle(g, s3, d3, sym, 8)
        # the exact Gauss-Seidel mode rebuilds its schedule for the new edges
        assert np.array_equal(g.pagerank(mode=gcgpu.PR_GS_EXACT, max_sweeps=3)[0], go.pagerank_gs_inmem(4))
        o32, _, _ = go.pagerank_jacobi(max_sweeps=10)
        assert np.abs(r1.astype(np.float64) - o32).sum() / np.abs(o32).sum() <= 1e-6
        assert np.array_equal(l1, go.cc()[0])


def test_updates_after_a_solve_and_nothing_to_delete():
    s, d = O.rmat_numpy(10, 8 << 10, seed=64)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
        g.pagerank(max_sweeps=5)  # builds and caches the PageRank plan
        e0 = g.num_edges
        g.delete_edges(np.array([1, 2], np.uint32), np.array([1, 2], np.uint32))  # self-loops: never present
        assert g.num_edges == e0
        g.add_edges(np.array([0, 3], np.uint32), np.array([3, 0], np.uint32))
        with gcgpu.Graph.from_edges(np.concatenate([s, [0, 3]]).astype(np.uint32),
                                    np.concatenate([d, [3, 0]]).astype(np.uint32), dedup=True) as ref:
            same_graph(g, ref)
            assert np.array_equal(g.pagerank(max_sweeps=5)[0], ref.pagerank(max_sweeps=5)[0])
