"""GPU parity of the device sharder (gcg_graph_from_edges) through the C ABI:
bit-exact against the reference's own sharder outputs (golden fixtures) and the
oracle restatement, plus edge cases."""
import hashlib

import numpy as np
import pytest

import gcgpu
import oracle as O
from conftest import golden_input, golden_names, load_golden

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check(z, key, arr):
    if key in z.files:
        assert np.array_equal(arr, z[key]), key
    else:
        assert sha(arr) == str(z[key + "_sha"]), key


@pytest.mark.parametrize("name", [n for n in golden_names() if "s20" not in n])
def test_sharder_matches_reference(name):
    z, spec = load_golden(name)
    s, d = golden_input(spec)
    sym = spec.get("sym", False)
    g_or = O.OracleGraph(s, d, symmetrise=sym)
    shard_keys = [k for k in z.files if k.startswith("intervals_")] or ["intervals_1"]
    for k in shard_keys:
        P = int(k.split("_")[1])
        with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=sym, nshards=P) as g:
            assert g.num_vertices == int(z["nv"]) and g.num_edges == int(z["ne"])
            if k in z.files:
                assert np.array_equal(g.intervals(), z[k])
                check(z, f"degrees_{P}", g.degrees())
            rp, col = g.csr(gcgpu.CSR_IN)
            assert np.array_equal(rp, g_or.in_rowptr) and np.array_equal(col, g_or.in_col)
            orp, ocol = g.csr(gcgpu.CSR_OUT)
            assert np.array_equal(orp, g_or.out_rowptr) and np.array_equal(ocol, g_or.out_col)
            if f"shard_sizes_{P}" in z.files:
                # shard p = out-edges (src-sorted) whose dst lies in interval p
                srcs = np.repeat(np.arange(g.num_vertices, dtype=np.uint32), np.diff(orp))
                lo, ss, dd = 0, [], []
                for hi in g.intervals():
                    m = (ocol >= lo) & (ocol <= hi)
                    ss.append(srcs[m])
                    dd.append(ocol[m])
                    lo = int(hi) + 1
                assert np.array_equal(np.array([len(x) for x in ss]), z[f"shard_sizes_{P}"])
                check(z, f"shard_src_{P}", np.concatenate(ss))
                check(z, f"shard_dst_{P}", np.concatenate(dd))


def test_intervals_many_shards_match_oracle():
    s, d = O.rmat_numpy(14, 16 << 14, seed=9)
    g_or = O.OracleGraph(s, d)
    for P in [1, 2, 3, 5, 16, 64, 1000, 20000]:
        with gcgpu.Graph.from_edges(s, d, dedup=True, nshards=P, out_csr=False) as g:
            assert np.array_equal(g.intervals(), g_or.intervals(P)), P


def test_device_and_host_inputs_agree():
    import torch
    s, d = O.rmat_numpy(15, 16 << 15, seed=4)
    ts, td = torch.from_numpy(s.astype(np.int32)).cuda(), torch.from_numpy(d.astype(np.int32)).cuda()
    with gcgpu.Graph.from_edges(s, d, dedup=True, nshards=8) as a, \
            gcgpu.Graph.from_edges(ts, td, dedup=True, nshards=8) as b:
        for w in (gcgpu.CSR_IN, gcgpu.CSR_OUT):
            ra, ca = a.csr(w)
            rb, cb = b.csr(w)
            assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
        assert np.array_equal(a.intervals(), b.intervals())


def test_device_generator_matches_host():
    import torch
    m = 1 << 20
    ts = torch.empty(m, dtype=torch.int32, device="cuda")
    td = torch.empty(m, dtype=torch.int32, device="cuda")
    gcgpu.generate_rmat(20, m, seed=5, src=ts, dst=td)
    hs, hd = gcgpu.generate_rmat(20, m, seed=5)
    assert np.array_equal(ts.cpu().numpy().view(np.uint32), hs)
    assert np.array_equal(td.cpu().numpy().view(np.uint32), hd)
    gcgpu.generate_er(123457, m, seed=6, src=ts, dst=td)
    es, ed = gcgpu.generate_er(123457, m, seed=6)
    assert np.array_equal(ts.cpu().numpy().view(np.uint32), es)


def test_multi_edges_kept_without_dedup():
    s = np.array([3, 1, 3, 1, 2, 2, 0, 3], np.uint32)
    d = np.array([1, 0, 1, 2, 2, 0, 3, 1], np.uint32)  # (2,2) self-loop dropped
    with gcgpu.Graph.from_edges(s, d, dedup=False) as g:
        rp, col = g.csr(gcgpu.CSR_IN)
        or_ = O.OracleGraph(s, d, dedup=False)
        assert np.array_equal(rp, or_.in_rowptr) and np.array_equal(col, or_.in_col)
        assert g.num_edges == 7


def test_symmetrise_dedup():
    s = np.array([0, 1, 1, 2, 5], np.uint32)
    d = np.array([1, 0, 2, 1, 4], np.uint32)
    with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=True) as g:
        rp, col = g.csr(gcgpu.CSR_IN)
        or_ = O.OracleGraph(s, d, symmetrise=True)
        assert np.array_equal(rp, or_.in_rowptr) and np.array_equal(col, or_.in_col)
        assert g.num_edges == 6


def test_empty_and_self_loop_only_graphs():
    e = np.zeros(0, np.uint32)
    with gcgpu.Graph.from_edges(e, e, nshards=4) as g:
        assert g.num_vertices == 1 and g.num_edges == 0
        assert g.intervals().tolist() == [0]
        r, st = g.pagerank(max_sweeps=3)
        assert r.shape == (1,) and abs(r[0] - 0.15) < 1e-7
    s = np.array([4, 4, 7], np.uint32)
    with gcgpu.Graph.from_edges(s, s) as g:
        assert g.num_edges == 0


def test_vertex_id_out_of_range_is_rejected():
    s = np.array([0, 5], np.uint32)
    d = np.array([1, 2], np.uint32)
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.Graph.from_edges(s, d, num_vertices=5)
    assert e.value.status == -1


def test_explicit_num_vertices_keeps_trailing_isolated():
    s = np.array([0, 1], np.uint32)
    d = np.array([1, 2], np.uint32)
    with gcgpu.Graph.from_edges(s, d, num_vertices=10, nshards=2) as g:
        assert g.num_vertices == 10
        rp, _ = g.csr()
        assert rp.tolist() == [0, 0, 1, 2, 2, 2, 2, 2, 2, 2, 2]


@pytest.mark.slow
def test_large_sort_matches_numpy():
    """2^22-vertex id space, 8M edges with duplicates: full 44-bit key sort."""
    s, d = O.rmat_numpy(22, 8 << 20, seed=21)
    with gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=True) as g:
        rp, col = g.csr(gcgpu.CSR_IN)
        keep = s != d
        k = np.unique((d[keep].astype(np.uint64) << np.uint64(32)) | s[keep].astype(np.uint64))
        assert g.num_edges == k.shape[0]
        assert np.array_equal(col, (k & np.uint64(0xFFFFFFFF)).astype(np.uint32))
        assert np.array_equal(np.diff(rp), np.bincount((k >> np.uint64(32)).astype(np.int64),
                                                       minlength=g.num_vertices).astype(np.uint32))
        orp, ocol = g.csr(gcgpu.CSR_OUT)
        k2 = np.unique((s[keep].astype(np.uint64) << np.uint64(32)) | d[keep].astype(np.uint64))
        assert np.array_equal(ocol, (k2 & np.uint64(0xFFFFFFFF)).astype(np.uint32))


def _same_graph(a, b):
    assert (a.num_vertices, a.num_edges) == (b.num_vertices, b.num_edges)
    assert a.info().has_out_csr == b.info().has_out_csr
    for w in ((gcgpu.CSR_IN, gcgpu.CSR_OUT) if a.info().has_out_csr else (gcgpu.CSR_IN,)):
        ra, ca = a.csr(w)
        rb, cb = b.csr(w)
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
    assert np.array_equal(a.degrees(), b.degrees())
    assert np.array_equal(a.intervals(), b.intervals())


@pytest.mark.parametrize("sym,dedup,pinned,out_csr,extra", [
    (False, True, True, True, 0), (True, True, True, False, 0), (False, False, False, True, 0),
    (False, True, True, False, 100), (True, False, True, False, 0)])
def test_host_edges_sorted_in_pieces_equal_one_sort(sym, dedup, pinned, out_csr, extra):
    """From 2^24 host edges on, the sharder sorts pieces of the edge list while
    later pieces are still being copied in, merges the sorted runs and fuses the
    last merge with the duplicate filter and the CSR decode (out-degrees are
    counted per piece when no out-CSR is built); the graph equals the one sorted
    in one piece from the same edges on the device. The last piece is ragged;
    R-MAT brings self-loops and duplicates; extra > 0 gives trailing isolated
    vertices through a caller-given vertex count."""
    import torch
    m = (1 << 24) + 12345
    s, d = O.rmat_numpy(20, m, seed=31)
    ts = torch.from_numpy(s.view(np.int32)).cuda()
    td = torch.from_numpy(d.view(np.int32)).cuda()
    if pinned:
        hs = torch.from_numpy(s.view(np.int32)).pin_memory()
        hd = torch.from_numpy(d.view(np.int32)).pin_memory()
    else:
        hs, hd = s, d
    nv = (1 << 20) + extra if extra else 0
    kw = dict(num_vertices=nv, dedup=dedup, symmetrise=sym, nshards=8, out_csr=out_csr)
    with gcgpu.Graph.from_edges(hs, hd, **kw) as a, gcgpu.Graph.from_edges(ts, td, **kw) as b:
        _same_graph(a, b)
        if not sym and dedup:
            keep = s != d
            k = np.unique((d[keep].astype(np.uint64) << np.uint64(32)) | s[keep].astype(np.uint64))
            assert a.num_edges == k.shape[0]
            _, col = a.csr(gcgpu.CSR_IN)
            assert np.array_equal(col, (k & np.uint64(0xFFFFFFFF)).astype(np.uint32))


def test_host_edges_in_pieces_reject_out_of_range_ids():
    m = 1 << 24
    s, d = O.rmat_numpy(20, m, seed=32)
    d[m - 7] = (1 << 20) + 5  # in the last piece
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.Graph.from_edges(s, d, num_vertices=1 << 20)
    assert e.value.status == -1
    # the same edges with a vertex count that admits the id build normally
    with gcgpu.Graph.from_edges(s, d, num_vertices=(1 << 20) + 6, dedup=True, out_csr=False) as g:
        assert g.num_vertices == (1 << 20) + 6
        assert g.degrees()[(1 << 20) + 5, 0] == 1  # the planted edge's destination


def test_largest_vertex_ids_are_rejected_not_wrapped():
    # id 2^32 - 1 would make max id + 1 wrap to 0; ids up to 2^32 - 2^26 - 1 are the limit
    for big in (0xFFFFFFFF, (1 << 32) - (1 << 26)):
        s = np.array([0, big], np.uint32)
        d = np.array([1, 2], np.uint32)
        with pytest.raises(gcgpu.GcgError) as e:
            gcgpu.Graph.from_edges(s, d)
        assert e.value.status == -6, big
