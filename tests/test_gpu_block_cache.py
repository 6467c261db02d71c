"""The library's block cache (gcg_cached_memory / gcg_release_cached_memory):
freed graph blocks are kept and handed to the next build of the same size, the
answers do not change, and releasing the cache gives every idle byte back."""
import numpy as np
import pytest

import gcgpu
import oracle as O

pytestmark = pytest.mark.gpu


def nl1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / np.abs(b).sum()


def build_and_solve(s, d):
    with gcgpu.Graph.from_edges(s, d, dedup=True, nshards=4) as g:
        r, st = g.pagerank(max_sweeps=30, tol=1e-9)
        return r, st.sweeps


def test_freed_blocks_are_reused_and_released():
    gcgpu.release_cached_memory()
    assert gcgpu.cached_memory() == (0, 0)
    s, d = O.rmat_numpy(14, 16 << 14, seed=71)
    r1, n1 = build_and_solve(s, d)
    dev1, host1 = gcgpu.cached_memory()
    assert dev1 > 0 and host1 > 0  # the graph's, plan's and workspace's blocks, the pinned flags
    r2, n2 = build_and_solve(s, d)
    assert np.array_equal(r1, r2) and n1 == n2
    # the same build asks for the same classes: the idle set is the same afterwards
    assert gcgpu.cached_memory() == (dev1, host1)
    released = gcgpu.release_cached_memory()
    assert released == dev1 + host1
    assert gcgpu.cached_memory() == (0, 0)
    r3, n3 = build_and_solve(s, d)
    assert np.array_equal(r1, r3) and n1 == n3


def test_recycled_blocks_give_the_oracle_answers():
    s, d = O.rmat_numpy(12, 8 << 12, seed=72)
    go = O.OracleGraph(s, d)
    ref, _, _ = go.pagerank_jacobi(max_sweeps=12)
    gs = O.OracleGraph(s, d, symmetrise=True)
    ref_cc, _ = gs.cc()
    for _ in range(3):  # the 2nd and 3rd builds run on recycled blocks
        with gcgpu.Graph.from_edges(s, d, dedup=True) as g:
            r, st = g.pagerank(max_sweeps=12)
            assert st.sweeps == 12 and nl1(r, ref) <= 1e-6
        with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=True) as g:
            lab, _ = g.connected_components()
            assert np.array_equal(lab, ref_cc)
