"""The warm-start oracle on its own (CPU): its analytic gradient against central
finite differences of its forward pass, and its features against their
definitions evaluated vertex by vertex on a small graph."""
import math

import numpy as np

import warm_oracle as W


def small_problem(seed=0, n=64):
    rng = np.random.default_rng(seed)
    params = np.zeros(W.NP)
    params[W.OW1:W.OB1] = rng.normal(0, math.sqrt(2 / 8), W.NH * W.NIN)
    params[W.OB1:W.OW2] = rng.normal(0, 0.1, W.NH)
    params[W.OW2:W.OB2] = rng.normal(0, math.sqrt(2 / 64), W.NH * W.NH)
    params[W.OB2:W.OW3] = rng.normal(0, 0.1, W.NH)
    params[W.OW3:W.OB3] = rng.normal(0, math.sqrt(1 / 64), W.NH)
    params[W.OB3] = 0.3
    norm = np.concatenate([rng.normal(0, 1, 8), rng.uniform(0.5, 2, 8)]).astype(np.float32)
    x = rng.normal(0, 1.5, (n, 8)).astype(np.float32)
    t = rng.normal(1, 1, n)
    return params, norm, x, t


def test_gradient_matches_finite_differences():
    params, norm, x, t = small_problem()
    g, _ = W.gradient(params, norm, x, t, rounding=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(np.arange(W.OW1, W.OB1), 12), rng.choice(np.arange(W.OB1, W.OW2), 6),
                          rng.choice(np.arange(W.OW2, W.OB2), 24), rng.choice(np.arange(W.OB2, W.OW3), 6),
                          rng.choice(np.arange(W.OW3, W.OB3), 8), [W.OB3]])
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (W.loss(p1, norm, x, t, rounding=False) - W.loss(p2, norm, x, t, rounding=False)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415927, 0.0, 65504.0, 1e-30], np.float32)
    r = W.bf16r(v)
    # every result is a BF16 value (low 16 bits zero) within half a BF16 ulp
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)
    assert np.all(np.abs(r - v) <= np.abs(v) * 2.0 ** -8 + 1e-38)
    # ties go to the even neighbour: 1 + 2^-8 lies halfway between 1 and 1 + 2^-7
    assert r[1] == 1.0
    assert W.bf16r(np.float32(1.0 + 3 * 2.0 ** -8)) == np.float32(1.0 + 2 * 2.0 ** -7)


def test_features_match_definitions():
    # a small directed graph as an in-edge CSR (sources per destination)
    nv = 11
    edges = [(0, 1), (2, 1), (3, 1), (1, 2), (4, 2), (1, 4), (5, 4), (6, 4), (7, 4), (4, 9), (1, 9), (9, 3)]
    src = np.array([s for s, _ in edges])
    dst = np.array([d for _, d in edges])
    order = np.lexsort((src, dst))
    src, dst = src[order], dst[order]
    indeg = np.bincount(dst, minlength=nv)
    outdeg = np.bincount(src, minlength=nv)
    rp = np.concatenate([[0], np.cumsum(indeg)])
    f = W.features(nv, rp, src, outdeg)
    B = W.vertex_bits(nv)
    assert B == 4
    for v in range(nv):
        nb = src[rp[v]:rp[v + 1]]
        exp = np.zeros(8)
        exp[0] = math.log1p(indeg[v])
        exp[1] = math.log1p(outdeg[v])
        if len(nb):
            exp[2] = np.mean([np.float32(math.log1p(indeg[u])) for u in nb])
            exp[3] = max(math.log1p(indeg[u]) for u in nb)
            exp[4] = math.log1p(sum(indeg[u] for u in nb))
        exp[5] = 1.0 / outdeg[v] if outdeg[v] else 0.0
        exp[6] = (v >> (B - 1)) & 1
        exp[7] = (v >> (B - 2)) & 1
        assert np.allclose(f[v], exp.astype(np.float32), rtol=1e-7, atol=0), (v, f[v], exp)
