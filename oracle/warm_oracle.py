"""ORACLE — test infrastructure only.

CPU restatement (numpy, float64 arithmetic) of the learned warm start: the
per-vertex degree features, the BF16 MLP's forward pass and its gradient. The
reference has no learned component (it starts PageRank from a constant,
example_apps/pagerank.cpp:80-85), so nothing in it pins these functions: the
gradient is pinned by central finite differences of this same forward pass
(with the BF16 roundings switched off, where the function is smooth), and the
features by direct evaluation of their definitions on small graphs. Only
tests/ may use this module, and only as the checker.

Definitions (the same as the C ABI's):
  features of v, L(u) = log(1 + indeg u):
    0 log(1+indeg v), 1 log(1+outdeg v), 2 mean L(u), 3 max L(u) (= log(1 + max
    indeg u)), 4 log(1 + sum indeg u) over in-neighbours u (0 without in-edges),
    5 1/outdeg v (0 without out-edges), 6/7 bits B-1, B-2 of v (B = bits of an id)
  network: x' = bf16((x - mean) * inv_std); h1 = bf16(relu(W1 x' + b1));
    h2 = relu(W2 h1 + b2); y = W3 . h2 + b3; W1, W2, W3 rounded to BF16.
  loss: mean((y - t)^2); gradients pass straight through the roundings.
  warm start: p = teleport*exp(y) with in-edges, teleport without; then p outside
    Z (no in-edges) scaled by the mass-stationary alpha (see mass_alpha).
"""
from __future__ import annotations

import numpy as np

NIN, NH = 8, 64
NP = NH * NIN + NH + NH * NH + NH + NH + 1
OW1 = 0
OB1 = OW1 + NH * NIN
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NH


def bf16r(x):
    """Round float32 values to the nearest BF16 value, ties to even (kept as float32)."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def vertex_bits(nv):
    b = 1
    while b < 32 and (1 << b) < nv:
        b += 1
    return b


def features(nv, in_rowptr, in_col, outdeg):
    """(nv, 8) float32 raw features from an in-edge CSR and the out-degrees."""
    rp = np.asarray(in_rowptr, np.int64)
    col = np.asarray(in_col, np.int64)
    indeg = np.diff(rp)
    outdeg = np.asarray(outdeg, np.int64)
    L = np.log1p(indeg.astype(np.float64)).astype(np.float32).astype(np.float64)
    f = np.zeros((nv, NIN), np.float64)
    f[:, 0] = np.log1p(indeg.astype(np.float64))
    f[:, 1] = np.log1p(outdeg.astype(np.float64))
    dst = np.repeat(np.arange(nv), indeg)
    if col.size:
        s = np.bincount(dst, weights=L[col], minlength=nv)
        mx = np.zeros(nv, np.int64)
        np.maximum.at(mx, dst, indeg[col])
        tot = np.bincount(dst, weights=indeg[col].astype(np.float64), minlength=nv)
        has = indeg > 0
        f[has, 2] = s[has] / indeg[has]
        f[has, 3] = np.log1p(mx[has].astype(np.float64))
        f[has, 4] = np.log1p(tot[has])
    nz = outdeg > 0
    f[nz, 5] = 1.0 / outdeg[nz]
    b = vertex_bits(nv)
    v = np.arange(nv, dtype=np.int64)
    f[:, 6] = (v >> (b - 1)) & 1 if b >= 1 else 0
    f[:, 7] = (v >> (b - 2)) & 1 if b >= 2 else 0
    return f.astype(np.float32)


def unpack(params):
    p = np.asarray(params, np.float64)
    return (p[OW1:OB1].reshape(NH, NIN), p[OB1:OW2], p[OW2:OB2].reshape(NH, NH), p[OB2:OW3], p[OW3:OB3],
            p[OB3])


def _inputs(norm, x, rounding):
    norm = np.asarray(norm, np.float32)
    xn = (np.asarray(x, np.float32) - norm[:NIN]) * norm[NIN:]  # float32, as the kernels compute it
    return (bf16r(xn) if rounding else xn).astype(np.float64)


def forward(params, norm, x, rounding=True, cache=False):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    if rounding:
        W1, W2, W3 = (bf16r(w.astype(np.float32)).astype(np.float64) for w in (W1, W2, W3))
    xh = _inputs(norm, x, rounding)
    a1 = xh @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    if rounding:
        h1 = bf16r(h1.astype(np.float32)).astype(np.float64)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ W3 + b3
    if cache:
        return y, (xh, a1, h1, a2, h2, W1, W2, W3)
    return y


def gradient(params, norm, x, t, rounding=True):
    """(gradient of mean((y - t)^2) w.r.t. the flat parameters, mean loss)."""
    y, (xh, a1, h1, a2, h2, W1, W2, W3) = forward(params, norm, x, rounding, cache=True)
    n = y.shape[0]
    err = y - np.asarray(t, np.float64)
    dy = 2.0 * err / n
    g = np.zeros(NP, np.float64)
    g[OW3:OB3] = h2.T @ dy
    g[OB3] = dy.sum()
    d2 = np.outer(dy, W3) * (a2 > 0)
    g[OW2:OB2] = (d2.T @ h1).ravel()
    g[OB2:OW3] = d2.sum(axis=0)
    d1 = (d2 @ W2) * (a1 > 0)
    g[OW1:OB1] = (d1.T @ xh).ravel()
    g[OB1:OW2] = d1.sum(axis=0)
    return g, float((err * err).mean())


def loss(params, norm, x, t, rounding=True):
    y = forward(params, norm, x, rounding)
    return float(((y - np.asarray(t, np.float64)) ** 2).mean())


def mass_alpha(p, indeg, outdeg, teleport=0.15, damping=0.85):
    """The factor that makes one Jacobi sweep keep the total rank when the
    predictions p outside Z (vertices without in-edges, fixed at teleport) are
    scaled by it: teleport*n + damping*(S - S_D) = S with S the total rank and
    S_D its part on vertices without out-edges."""
    p = np.asarray(p, np.float64)
    Z = np.asarray(indeg) == 0
    D = np.asarray(outdeg) == 0
    M = p[~Z].sum()
    MD = p[~Z & D].sum()
    num = teleport * (p.size - (1 - damping) * Z.sum() - damping * (Z & D).sum())
    den = (1 - damping) * M + damping * MD
    return num / den if den > 0 and num > 0 else 1.0
