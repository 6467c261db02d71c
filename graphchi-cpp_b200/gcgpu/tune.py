"""Launch-configuration report of the Jacobi PageRank edge phase on a seeded
R-MAT graph: for each configuration, the edge phase and the whole sweep per
sweep (CUDA events on the graph's stream, best of three 20-sweep runs) and the
edge phase's share of the HBM roofline (8E + 16V bytes per sweep against the
measured copy bandwidth in MEASURED_PEAKS.json, else 6650 GB/s). Every
configuration computes the same sums in the same order except source tiers
(tiers > 1), whose rows add per-tier partial sums.

    python -m gcgpu.tune --scale 24 [--tiers 1 2 3 4] [--hub 41724 32768]

With --batch LO HI it reports the many-graph persistent launch instead: 64
graphs, vertex counts log-uniform in [LO, HI] (seeded), alternating
Erdos-Renyi (mean degree 8) and R-MAT (edge factor 8), solved to 1e-8 in one
launch for each --hub value, against one gcg_pagerank solve per graph.

With --ppr K it reports batched personalised PageRank on the R-MAT graph of
each --scale (seed + 6): K seeded sources to 1e-8 in one gcg_ppr_batched call
(best of two), against E(4 + 4k) + 12Vk bytes per sweep over the k sources still
iterating. With --cc it reports connected components on the symmetrised R-MAT
graph of each --scale (best of three calls) against one streaming pass over the
graph (8E + 12V bytes). With --tc it reports triangle counting (degree
ranking, orientation, count; per-rank counts into device memory) on the
symmetrised R-MAT graph of each --scale (best of three calls).

(run with graphchi-cpp_b200 on PYTHONPATH)."""
from __future__ import annotations

import argparse
import json
import os


def peak_gbs():
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    try:
        with open(os.path.join(root, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def batch_report(lo, hi, hubs, peak):
    import math
    import numpy as np
    import torch
    import gcgpu
    rng = np.random.default_rng(5)
    ns = np.exp(rng.uniform(math.log(lo), math.log(hi), 64)).astype(int)
    gs = []
    for i, nn in enumerate(ns):
        if i % 2 == 0:
            mm = 8 * int(nn)
            s = torch.empty(mm, dtype=torch.int32, device="cuda")
            d = torch.empty_like(s)
            gcgpu.generate_er(int(nn), mm, 100 + i, s, d)
            gs.append(gcgpu.Graph.from_edges(s, d, num_vertices=int(nn), dedup=True, out_csr=False))
        else:
            sc = max(1, round(math.log2(nn)))
            s = torch.empty(8 << sc, dtype=torch.int32, device="cuda")
            d = torch.empty_like(s)
            gcgpu.generate_rmat(sc, 8 << sc, 0.57, 0.19, 0.19, seed=100 + i, src=s, dst=d)
            gs.append(gcgpu.Graph.from_edges(s, d, num_vertices=1 << sc, dedup=True, out_csr=False))
    seq = 0.0
    for g in gs:
        o = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")
        g.pagerank(max_sweeps=1000, tol=1e-8, out=o)
        seq += g.pagerank(max_sweeps=1000, tol=1e-8, out=o)[1].device_ms
    with gcgpu.Batch(gs) as b:
        allr = torch.empty(int(b.offsets[-1]), dtype=torch.float32, device="cuda")
        for hub in hubs:
            b.set_config(hub, 0)
            b.pagerank(max_sweeps=1000, tol=1e-8, out=allr)
            best = min((b.pagerank(max_sweeps=1000, tol=1e-8, out=allr) for _ in range(3)),
                       key=lambda x: x[3].device_ms)
            st, gsw = best[3], best[1]
            byt = float(sum(int(n) * (8.0 * g.num_edges + 16.0 * g.num_vertices) for n, g in zip(gsw, gs)))
            print(json.dumps({"batch": [lo, hi], "graphs": 64, "vertices": int(b.offsets[-1]),
                              "edges": int(sum(g.num_edges for g in gs)), "hub": hub,
                              "max_sweeps": int(gsw.max()), "ms_one_launch": round(st.device_ms, 2),
                              "ms_one_solve_per_graph": round(seq, 2), "speedup": round(seq / st.device_ms, 2),
                              "frac_of_hbm": round(byt / st.device_ms / 1e6 / peak, 3)}), flush=True)
    for g in gs:
        g.free()


def ppr_report(scale, ef, seed, k, peak):
    import numpy as np
    import torch
    import gcgpu
    m = ef << scale
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    gcgpu.generate_rmat(scale, m, 0.57, 0.19, 0.19, seed=seed + 6, src=s, dst=d)
    with gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=False) as g:
        del s, d
        n, E = g.num_vertices, g.num_edges
        src = np.random.default_rng(3).integers(0, n, k).astype(np.uint32)
        mat = torch.empty((n, k), dtype=torch.float32, device="cuda")
        runs = []
        for _ in range(2):
            wl = np.zeros(2 * 1000, np.uint64)
            st = g.ppr_batched(src, max_sweeps=1000, tol=1e-8, teleport=0.15, out=mat, work_log=wl)[1]
            runs.append((st.device_ms, st.sweeps, wl))
        ms, sweeps, wl = min(runs, key=lambda r: r[0])
        upd, gat = int(wl[2 * sweeps - 2]), int(wl[2 * sweeps - 1])
        byt = 4.0 * E * sweeps + 4.0 * gat + 12.0 * upd
        print(json.dumps({"ppr": {"scale": scale, "vertices": n, "edges": E, "sources": k, "sweeps": sweeps,
                                  "source_sweeps": gat // max(1, E), "ms": round(ms, 2),
                                  "algorithmic_bytes": byt, "frac_of_hbm": round(byt / ms / 1e6 / peak, 3)}}),
              flush=True)


def cc_report(scale, ef, seed, peak):
    import torch
    import gcgpu
    m = ef << scale
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    gcgpu.generate_rmat(scale, m, 0.57, 0.19, 0.19, seed=seed, src=s, dst=d)
    with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=True, out_csr=False) as g:
        del s, d
        lab = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
        g.connected_components(out=lab)
        ms = min(g.connected_components(out=lab)[1].device_ms for _ in range(3))
        byt = 8.0 * g.num_edges + 12.0 * g.num_vertices
        print(json.dumps({"cc": {"scale": scale, "vertices": g.num_vertices, "directed_edges": g.num_edges,
                                 "ms": round(ms, 3), "one_pass_bytes": byt,
                                 "frac_of_one_pass_at_hbm": round(byt / ms / 1e6 / peak, 3)}}), flush=True)


def tc_report(scale, ef, seed):
    import torch
    import gcgpu
    m = ef << scale
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    gcgpu.generate_rmat(scale, m, 0.57, 0.19, 0.19, seed=seed, src=s, dst=d)
    with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=True, out_csr=False) as g:
        del s, d
        per = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
        tri = g.triangle_count(per_rank=per, vertexmap=None)[0]
        ms = min(g.triangle_count(per_rank=per, vertexmap=None)[3].device_ms for _ in range(3))
        print(json.dumps({"tc": {"scale": scale, "vertices": g.num_vertices, "directed_edges": g.num_edges,
                                 "triangles": tri, "ms": round(ms, 3)}}), flush=True)


def main():
    import torch
    import gcgpu
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, nargs="+", default=[24])
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--hub", type=int, nargs="+", default=[41724])
    ap.add_argument("--tiers", type=int, nargs="+", default=[1])
    ap.add_argument("--batch", type=float, nargs=2, default=None, metavar=("LO", "HI"))
    ap.add_argument("--ppr", type=int, default=0, metavar="K")
    ap.add_argument("--cc", action="store_true")
    ap.add_argument("--tc", action="store_true")
    args = ap.parse_args()
    peak = peak_gbs()
    if args.batch:
        batch_report(args.batch[0], args.batch[1], args.hub, peak)
        return
    if args.ppr or args.cc or args.tc:
        for scale in args.scale:
            if args.ppr:
                ppr_report(scale, args.ef, args.seed, args.ppr, peak)
            if args.cc:
                cc_report(scale, args.ef, args.seed, peak)
            if args.tc:
                tc_report(scale, args.ef, args.seed)
        return
    for scale in args.scale:
        m = args.ef << scale
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        gcgpu.generate_rmat(scale, m, 0.57, 0.19, 0.19, seed=args.seed, src=s, dst=d)
        g = gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=False)
        del s, d
        torch.cuda.empty_cache()
        out = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")
        E, V = g.num_edges, g.num_vertices
        for hub in args.hub:
            for t in args.tiers:
                g.pagerank_config(hub, 1)
                g.pagerank_tiers(t)
                g.pagerank(max_sweeps=4, out=out)
                best = None
                for _ in range(3):
                    _, st = g.pagerank(max_sweeps=20, out=out, time_sweeps=True)
                    e = st.sweep_kernel_ms / st.timed_sweeps
                    if best is None or e < best[0]:
                        best = (e, st.device_ms / st.sweeps)
                print(json.dumps({"scale": scale, "vertices": V, "edges": E, "hub": hub, "tiers": t,
                                  "edge_phase_us": round(best[0] * 1e3, 1), "sweep_us": round(best[1] * 1e3, 1),
                                  "edge_frac_of_hbm": round((8 * E + 16 * V) / best[0] / 1e6 / peak, 3)}),
                      flush=True)
        g.free()


if __name__ == "__main__":
    main()
