"""Learned warm start: training data from the engine's own PageRank solves,
training on the device, and evaluation against the uniform start.

    python -m gcgpu.warm train --graphs 200 --scales 18-22 --out model.npz
    python -m gcgpu.warm eval --model model.npz --scale 24 --graphs 10

Every step runs through libgcgpu (device R-MAT generator, device sharder,
Jacobi PageRank, the feature / training / inference kernels); this module only
orders the calls and holds the samples.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import Graph, Mlp, generate_rmat

TELEPORT = 0.15
DAMPING = 0.85
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warm_start_rmat.npz")


def _device_edges(scale, m, a, b, c, seed):
    import torch
    src = torch.empty(m, dtype=torch.int32, device="cuda")
    dst = torch.empty(m, dtype=torch.int32, device="cuda")
    generate_rmat(scale, m, a, b, c, seed, src, dst)
    return src, dst


def jittered_abc(rng, jitter=0.05):
    """R-MAT a/b/c/d = 0.57/0.19/0.19/0.05, each moved by up to +-jitter, renormalised."""
    p = np.array([0.57, 0.19, 0.19, 0.05]) + rng.uniform(-jitter, jitter, 4)
    p = np.clip(p, 0.01, None)
    p /= p.sum()
    return float(p[0]), float(p[1]), float(p[2])


def rmat_graph(scale, seed, abc=(0.57, 0.19, 0.19), ef=16) -> Graph:
    src, dst = _device_edges(scale, ef << scale, *abc, seed)
    return Graph.from_edges(src, dst, dedup=True, out_csr=False)


def samples(g: Graph, max_samples=None, rng=None, tol=1e-8):
    """(features, targets) of the vertices with in-edges: target = log(rank / teleport)
    of the engine's Jacobi PageRank run to tol. Vertices without in-edges are left out
    (the warm start sets them to their exact rank)."""
    import torch
    n = g.num_vertices
    x = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    g.warm_features(x)
    r = torch.empty(n, dtype=torch.float32, device="cuda")
    g.pagerank(max_sweeps=1000, tol=tol, teleport=TELEPORT, damping=DAMPING, out=r)
    keep = torch.nonzero(x[:, 0] > 0).squeeze(1)
    if max_samples is not None and keep.numel() > max_samples:
        gen = torch.Generator(device="cpu")
        gen.manual_seed(int(rng.integers(1 << 62)) if rng is not None else 0)
        keep = keep[torch.randperm(keep.numel(), generator=gen)[:max_samples].to(keep.device)]
    t = torch.log(r[keep].double() / TELEPORT).float()
    return x[keep].contiguous(), t.contiguous()


def build_training_set(ngraphs=200, scales=(18, 22), per_graph=65536, seed=1, jitter=0.05, log=None):
    """Samples from ngraphs seeded R-MAT graphs, scale uniform in [scales[0], scales[1]],
    a/b/c/d jittered. Returns device tensors (x, t)."""
    import torch
    rng = np.random.default_rng(seed)
    xs, ts = [], []
    for i in range(ngraphs):
        scale = int(rng.integers(scales[0], scales[1] + 1))
        abc = jittered_abc(rng, jitter)
        gseed = int(rng.integers(1 << 40))
        with rmat_graph(scale, gseed, abc) as g:
            x, t = samples(g, per_graph, rng)
        xs.append(x)
        ts.append(t)
        if log:
            log(f"graph {i}: scale {scale} abc {abc[0]:.3f}/{abc[1]:.3f}/{abc[2]:.3f} samples {t.numel()}")
    return torch.cat(xs), torch.cat(ts)


def train(x, t, epochs=8, batch=4096, lr=2e-3, seed=1, model_seed=1, rank_power=0.5) -> tuple:
    """One model: normalisation from the samples, then minibatch Adam on a
    resampling of the samples with probability proportional to (rank/teleport)^rank_power
    (high-rank vertices carry the slow modes of the iteration)."""
    import torch
    m = Mlp(seed=model_seed)
    m.fit_normalisation(x)
    if rank_power:
        w = torch.exp(rank_power * t.double())
        gen = torch.Generator(device=t.device)
        gen.manual_seed(int(seed))
        idx = torch.multinomial(w / w.sum(), t.numel(), replacement=True, generator=gen)
        x, t = x[idx].contiguous(), t[idx].contiguous()
    losses = m.train(x, t, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return m, losses


def validation_specs(n=3, scale=20, seed=4242):
    rng = np.random.default_rng(seed)
    return [(scale, int(rng.integers(1 << 40)), jittered_abc(rng)) for _ in range(n)]


def train_selected(x, t, candidates=4, val=None, log=None, **kw):
    """Trains `candidates` models (different seeds) and keeps the one whose warm
    start needs the fewest Jacobi sweeps to 1e-8 on the validation graphs (the
    uniform-start iteration is the reference for each). Returns (model, losses, report)."""
    val = validation_specs() if val is None else val
    graphs = [rmat_graph(*sp) for sp in val]
    best = None
    report = []
    try:
        for c in range(candidates):
            m, losses = train(x, t, seed=1 + c, model_seed=1 + c, **kw)
            sweeps = [evaluate(g, m)["sweeps_warm"] for g in graphs]
            report.append({"candidate": c, "loss": float(losses[-1]), "val_sweeps": sweeps})
            if log:
                log(json.dumps(report[-1]))
            if best is None or sum(sweeps) < best[0]:
                if best is not None:
                    best[1].free()
                best = (sum(sweeps), m, losses)
            else:
                m.free()
    finally:
        for g in graphs:
            g.free()
    return best[1], best[2], report


def evaluate(g: Graph, m: Mlp, tol=1e-8, repeats=1):
    """Plain (uniform start) vs warm-started Jacobi PageRank to the same residual.
    Times are device times (CUDA events); the warm time includes the features and
    the network."""
    import torch
    n = g.num_vertices
    r0 = torch.empty(n, dtype=torch.float32, device="cuda")
    r1 = torch.empty(n, dtype=torch.float32, device="cuda")
    init = torch.empty(n, dtype=torch.float32, device="cuda")
    best = None
    for _ in range(repeats):
        _, sp = g.pagerank(max_sweeps=1000, tol=tol, teleport=TELEPORT, damping=DAMPING, out=r0)
        _, wms = g.warm_start_rank(m, TELEPORT, DAMPING, out=init)
        _, sw = g.pagerank(max_sweeps=1000, tol=tol, teleport=TELEPORT, damping=DAMPING, init_rank=init, out=r1)
        rec = {"sweeps_plain": sp.sweeps, "sweeps_warm": sw.sweeps, "ms_plain": sp.device_ms,
               "ms_warm": wms + sw.device_ms, "ms_warm_start": wms,
               "residual_plain": sp.residual, "residual_warm": sw.residual}
        if best is None or rec["ms_warm"] + rec["ms_plain"] < best["ms_warm"] + best["ms_plain"]:
            best = rec
    d = (r0.double() - r1.double()).abs().sum() / r0.double().abs().sum()
    best["l1_between"] = float(d)
    e0 = (init.double() - r0.double()).abs().sum() / r0.double().abs().sum()
    best["init_l1_error"] = float(e0)
    best["uniform_l1_error"] = float((1.0 - r0.double()).abs().sum() / r0.double().abs().sum())
    return best


def _main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--graphs", type=int, default=200)
    tr.add_argument("--scales", default="18-22")
    tr.add_argument("--per-graph", type=int, default=65536)
    tr.add_argument("--epochs", type=int, default=8)
    tr.add_argument("--batch", type=int, default=4096)
    tr.add_argument("--lr", type=float, default=2e-3)
    tr.add_argument("--seed", type=int, default=1)
    tr.add_argument("--candidates", type=int, default=4)
    tr.add_argument("--val-graphs", type=int, default=3)
    tr.add_argument("--val-scale", type=int, default=20)
    tr.add_argument("--out", default=MODEL_PATH)
    ev = sub.add_parser("eval")
    ev.add_argument("--model", default=MODEL_PATH)
    ev.add_argument("--scale", type=int, default=24)
    ev.add_argument("--graphs", type=int, default=10)
    ev.add_argument("--seed", type=int, default=1000)
    ev.add_argument("--repeats", type=int, default=2)
    a = ap.parse_args()
    if a.cmd == "train":
        lo, hi = (int(v) for v in a.scales.split("-"))
        t0 = time.time()
        x, t = build_training_set(a.graphs, (lo, hi), a.per_graph, a.seed, log=print)
        t1 = time.time()
        m, losses, rep = train_selected(x, t, a.candidates, validation_specs(a.val_graphs, a.val_scale), log=print,
                                        epochs=a.epochs, batch=a.batch, lr=a.lr)
        t2 = time.time()
        m.save(a.out)
        print(json.dumps({"samples": int(t.numel()), "data_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2),
                          "epoch_loss": [round(float(v), 5) for v in losses], "out": a.out}))
    else:
        m = Mlp.load(a.model)
        rng = np.random.default_rng(a.seed)
        rows = []
        for i in range(a.graphs):
            abc = jittered_abc(rng)
            with rmat_graph(a.scale, int(rng.integers(1 << 40)), abc) as g:
                rec = evaluate(g, m, repeats=a.repeats)
            rows.append(rec)
            print(json.dumps(rec))
        sp = sum(r["ms_plain"] for r in rows)
        sw = sum(r["ms_warm"] for r in rows)
        print(json.dumps({"graphs": len(rows), "ms_plain_total": round(sp, 3), "ms_warm_total": round(sw, 3),
                          "speedup": round(sp / sw, 4),
                          "sweeps_plain_mean": float(np.mean([r["sweeps_plain"] for r in rows])),
                          "sweeps_warm_mean": float(np.mean([r["sweeps_warm"] for r in rows]))}))


if __name__ == "__main__":
    _main()
