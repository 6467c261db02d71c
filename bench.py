#!/usr/bin/env python
"""PageRank GTEPS on one B200: R-MAT scale 24, edge factor 16, run to normalised
L1 residual <= 1e-8 (damping 0.85, FP32 values, FP64 residual).

One step = one full PageRank solve (Jacobi, uniform init) to the tolerance on
the device-resident graph. Synthetic input: the seeded R-MAT generator of
csrc/gcg_rng.h (a/b/c/d = .57/.19/.19/.05), duplicates and self-loops removed by
the device sharder, 64 vertex intervals.

  value      GTEPS = edges x sweeps / device time, inputs resident in HBM
  e2e        same metric through the C ABI with host buffers: pinned host edge
             arrays -> gcg_graph_from_edges (H2D + device sharder) ->
             gcg_pagerank -> ranks to host, every step
  roofline   the main sweep kernel (k_pr_edges): 8E+16V algorithmic bytes per
             launch / its CUDA-event launch time, against measured HBM copy GB/s
  oracle_check  the solve's error against the oracle on the same graph, built
             independently on the host: FP64 Jacobi to residual 1e-12 and the
             FP32 iteration to the same tolerance (normalised L1)
  cpu_baseline  that FP32 oracle iteration (a port of the reference's
             bulk-synchronous PageRank) timed to the tolerance on all host cores
  extras     the other rows against their plain methods: the bit-exact
             vertex-API program to the tolerance, connected components (+
             triangles) on symmetrised R-MAT, the learned warm start, batched
             personalised PageRank, 64 uneven graphs in one persistent launch

--impl reference times the reference's own PageRank app (oracle/_ref/pagerank,
built from the reference sources, its default in-memory vertex program) on the
same scale-24 graph, one step = one of its iterations (rank 0; other ranks exit).
Under torchrun (N > 1) every rank solves its own replica (the path does not
shard: replicas only); value sums the ranks' edges over the max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "graphchi-cpp_b200"))

METRIC = "PageRank GTEPS (R-MAT scale 24, ef 16, to L1 residual 1e-8)"
UNIT = "GTEPS"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_pr_edges
# launch per edge at R-MAT scale 24: 1.130 GB + 15.7 MB for 263,430,537 edges in
# one ncu capture of the full-size workload (ncu --set full --clock-control none
# -k regex:"k_pr_(edges|vertex)" -s 4 -c 2 python bench.py --steps 1 --warmup 1
# --e2e-steps 0 --e2e-warmup 0 --no-extras --no-cpu-baseline --no-oracle-check);
# traffic scales with the edges swept.
TRAFFIC_BYTES_PER_EDGE = 4.35


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# Sweeps the vertex-API in-memory program (example_apps/pagerank.cpp:121-146,
# Gauss-Seidel in vertex id order) needs to reach normalised L1 residual 1e-8 on
# the R-MAT scale-24 ef-16 seed-1 graph: 51, from the oracle's restatement of the
# program with per-sweep tracking (orc_pagerank_gs_track; 96 s on one core);
# the extras' gs_exact row measures it live with the bit-exact GCG_PR_GS_EXACT
# mode. The reference app has a fixed iteration count and no residual; its time
# to the tolerance is its iteration time times this count.
GS_SWEEPS_TO_TOL_RMAT24 = 51


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def reference_iterations(scale, ef, seed, warmup, steps, threads, engine_inmem=False):
    """Runs the reference's own PageRank app (oracle/_ref/pagerank, built from
    example_apps/pagerank.cpp) on the R-MAT graph of the headline workload, made
    by the oracle's restatement of the generator (no library code on this path):
    the edge list is written, the reference shards it (convert_if_notexists,
    nshards auto), then runs warmup + steps + 2 iterations with its default
    configuration (membudget 800 MB: the in-memory vertex program). With
    engine_inmem, one shard and a 30 GB budget instead: the engine's in-memory mode
    (graphchi_engine.hpp:299-301, 465-530), every vertex and edge held in RAM. The engine's
    log line "Start iteration: k" (graphchi_engine.hpp:780; "In-memory mode:
    Iteration k starts" with a single shard, :468) arrives on stderr as iteration
    k starts; the time between two of them is one iteration (one sweep over every
    in-edge).
    Iteration 0 (initialisation) and the next `warmup` are not timed."""
    O = _oracle()
    if not O.ref_available():
        raise RuntimeError("oracle/_ref is not built")
    import re
    t0 = time.perf_counter()
    s, d = O.rmat_edges(scale, ef << scale, seed=seed)
    cs, cd = O.canonical_edges(s, d, symmetrise=False, dedup=True)
    del s, d
    E, V = int(cs.shape[0]), O.num_vertices(cs, cd)
    niters = warmup + steps + 2
    with O.RefWorkdir(prefix="gcg_bench_ref_") as w:
        el = w.file("g.el")
        O.write_edgelist(el, cs, cd)
        del cs, cd
        prep_s = time.perf_counter() - t0
        args = [os.path.join(O.REF_DIR, "pagerank"), "file", el, "filetype", "edgelist", "niters", str(niters),
                "nshards", "1" if engine_inmem else "auto", "execthreads", str(threads), "loadthreads", str(threads)]
        if engine_inmem:
            args += ["membudget_mb", "30000"]
        env = dict(os.environ, GRAPHCHI_ROOT=O.REF_DIR, OMP_NUM_THREADS=str(threads))
        starts, out_lines = {}, []
        t1 = time.perf_counter()
        p = subprocess.Popen(args, env=env, cwd=w.path, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        reader = threading.Thread(target=lambda: out_lines.extend(p.stdout), daemon=True)
        reader.start()
        err_tail = []
        for line in p.stderr:
            t = time.perf_counter()
            # the shard-streaming engine's line, or the single-shard in-memory mode's
            m = re.search(r"Start iteration: (\d+)", line) or re.search(r"In-memory mode: Iteration (\d+) starts",
                                                                          line)
            if m:
                starts[int(m.group(1))] = t
            err_tail = (err_tail + [line])[-20:]
        rc = p.wait()
        reader.join(timeout=10)
        wall = time.perf_counter() - t1
        if rc != 0:
            raise RuntimeError(f"reference pagerank failed ({rc}): {''.join(err_tail)[-500:]}")
        out = "".join(out_lines) + "".join(err_tail)
        runtime = O.ref_runtime(out)
    timed = list(range(1 + warmup, 1 + warmup + steps))
    if any(k + 1 not in starts or k not in starts for k in timed):
        raise RuntimeError(f"iteration start lines missing: saw {sorted(starts)[:5]}... of {niters}")
    it_s = [starts[k + 1] - starts[k] for k in timed]
    shard_s = starts[0] - t1 if 0 in starts else None
    return {"edges": E, "vertices": V, "iteration_s": it_s, "gteps": [E / t / 1e9 for t in it_s],
            "prep_s": prep_s, "shard_and_load_s": shard_s, "run_wall_s": wall, "engine_runtime_s": runtime,
            "niters": niters}


def oracle_check(scale, ef, seed, tol, gpu_rank, gpu_sweeps, threads):
    """The headline solve against the oracle on the same graph, built on the host
    by the oracle alone (generator restatement, canonical in-CSR): the FP64
    Jacobi iteration to residual 1e-12 (its error to the fixed point is below
    1e-11) and the FP32 iteration (the reference's bulk-synchronous PageRank
    restated) to the same tolerance as the GPU; normalised L1 of the GPU's ranks
    against each. The FP32 run is timed: it is the CPU baseline on this workload."""
    import numpy as np
    O = _oracle()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    t0 = time.perf_counter()
    s, d = O.rmat_edges(scale, ef << scale, seed=seed)
    go = O.OracleGraph.in_csr_only(s, d)
    del s, d
    build_s = time.perf_counter() - t0
    r = np.asarray(gpu_rank, np.float64)

    def nl1(x):
        x = np.asarray(x, np.float64)
        return float(np.abs(r - x).sum() / np.abs(x).sum())

    t0 = time.perf_counter()
    f64, n64, log64 = go.pagerank_jacobi_f64_mt(max_sweeps=3000, tol=1e-12)
    f64_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    o32, n32, log32 = go.pagerank_jacobi_mt(max_sweeps=3000, tol=tol)
    f32_s = time.perf_counter() - t0
    return {"graph": f"rmat{scale}_ef{ef}_seed{seed}", "vertices": go.nv, "edges": go.ne,
            "fp64_oracle_l1": nl1(f64), "fp64_sweeps": n64, "fp64_last_residual": float(log64[-1]),
            "fp32_oracle_l1": nl1(o32), "fp32_sweeps": n32, "gpu_sweeps": gpu_sweeps,
            "fp32_oracle_vs_fp64_l1": float(np.abs(o32.astype(np.float64) - f64).sum() / np.abs(f64).sum()),
            "tolerance_l1": 1e-6, "pass": nl1(f64) <= 1e-6 and nl1(o32) <= 1e-6,
            "host_build_s": build_s, "fp64_s": f64_s, "fp32_s": f32_s, "threads": threads,
            "note": "oracle/oracle.c: graph from the generator restatement (self-loops dropped, duplicates "
                    "removed), Jacobi 0.15 + 0.85 sum over in-neighbours' rank / outdeg, init 1"}


def max_over_ranks(x, world, device):
    """The largest x over all ranks: the slowest replica sets the job's time
    (identity on one rank)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gteps(edges_per_rank, world, seconds):
    """GTEPS of the whole job: every rank runs the same workload (replicas), so the
    edges of all ranks over the slowest rank's time."""
    return edges_per_rank * world / seconds / 1e9


def run_reference(args, rank, world):
    """The reference arm: the reference's own PageRank app on the headline graph,
    twice. The line's value is the engine's in-memory mode (one shard, every vertex
    and edge in RAM; at the headline size 3.4x faster than the default); the run
    with the default configuration (membudget 800 MB, 11 shards streamed from the
    page cache at scale 24) is reported beside it in cpu_baseline.default_budget,
    a bounded sample of at most 3 timed iterations (--no-ref-inmem: that run alone,
    with all the steps, as the value)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    headline_graph = args.scale == 24 and args.ef == 16 and args.seed == 1
    runs = {}
    for mode in (("default",) if args.no_ref_inmem else ("inmem", "default")):
        # the default-budget run beside the in-memory one is a bounded sample (its
        # iterations take ~3.4x as long): at most 3 timed iterations after 1 warm-up
        secondary = mode == "default" and not args.no_ref_inmem
        w, k = (min(args.warmup, 1), min(args.steps, 3)) if secondary else (args.warmup, args.steps)
        try:
            runs[mode] = reference_iterations(args.scale, args.ef, args.seed, w, k, threads,
                                              engine_inmem=mode == "inmem")
            runs[mode]["steps"] = k
        except Exception as e:  # noqa: BLE001
            runs[mode] = e
    primary = "inmem" if isinstance(runs.get("inmem"), dict) else "default"
    rec = runs[primary]
    if not isinstance(rec, dict):
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {rec}"[:300]}))
        return
    E = rec["edges"]

    def summary(r):
        t = sum(r["iteration_s"])
        out = {"value": E * r["steps"] / t / 1e9, "unit": UNIT, "iteration_s": r["iteration_s"],
               "shard_and_load_s": r["shard_and_load_s"], "input_prep_s": r["prep_s"],
               "engine_runtime_s": r["engine_runtime_s"]}
        if GS_SWEEPS_TO_TOL_RMAT24 and headline_graph:
            out["time_to_tol_s"] = t / r["steps"] * GS_SWEEPS_TO_TOL_RMAT24
            out["time_to_tol_note"] = (
                f"mean iteration time x {GS_SWEEPS_TO_TOL_RMAT24} Gauss-Seidel sweeps to residual {args.tol:g} "
                "(the sweeps this program needs, measured by the bit-exact GCG_PR_GS_EXACT mode)")
        return out

    main = summary(rec)
    v = main["value"]
    tot = sum(rec["iteration_s"])
    how = ("the engine's in-memory mode: nshards 1, membudget_mb 30000, every vertex and edge in RAM"
           if primary == "inmem" else "default membudget 800 MB, shards streamed from the page cache")
    sample = (f"oracle/_ref/pagerank (example_apps/pagerank.cpp: the in-memory vertex program, Gauss-Seidel in "
              f"vertex id order; {how}) on R-MAT scale {args.scale} ef {args.ef} seed {args.seed} ({E} edges "
              f"after dedup{', the headline graph' if headline_graph else ''}), {rec['niters']} iterations in one run; one step = one iteration "
              f"timed between the engine's iteration-start log lines; iteration 0 and {args.warmup} warm-up "
              f"iterations untimed; sharding untimed")
    cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample}
    cpu.update({k: main[k] for k in main if k not in ("value", "unit")})
    if primary == "inmem":
        d = runs["default"]
        cpu["default_budget"] = (dict(summary(d), config="membudget_mb 800 (the default), nshards auto")
                                 if isinstance(d, dict) else {"unavailable": f"default run failed: {d}"[:300]})
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"pagerank_rmat{args.scale}_ef{args.ef}_to_{args.tol:g}", "vertices": rec["vertices"],
                   "edges": E, "step": "one PageRank iteration (sweep) of the reference engine",
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_extras(args):
    """The other rows of the workload, each against its plain method on the same
    device (all device times by CUDA events; rank 0 of a 1-GPU run):
      cc            connected components, symmetrised R-MAT scale 24 (and 20) + triangles at 20
      warm_start    learned warm start vs uniform start to 1e-8 on the scale-24 graph
      batched_ppr   256 personalised sources at once vs single-source solves, scale 22
      batched_graphs 64 uneven graphs (10k-2M vertices, ER mean degree 8 / R-MAT) in one
                    autotuned, graph-captured persistent launch vs one solve per graph"""
    import math
    import numpy as np
    import torch
    import gcgpu
    import gcgpu.warm as gw
    out = {}
    peak, _ = load_peaks()

    def dev_edges(scale, m, seed, abc=(0.57, 0.19, 0.19)):
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty(m, dtype=torch.int32, device="cuda")
        gcgpu.generate_rmat(scale, m, *abc, seed=seed, src=s, dst=d)
        return s, d

    # ---- the device sharder on the headline input (edges already on the device) ----
    m = args.ef << args.scale
    s, d = dev_edges(args.scale, m, args.seed)
    t_build = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gb = gcgpu.Graph.from_edges(s, d, dedup=True, nshards=args.nshards, out_csr=False)
        torch.cuda.synchronize()
        t_build.append((time.perf_counter() - t0) * 1e3)
        gb.free()
    del s, d
    bms = min(t_build[1:])
    # the LSD sort of (dst, src) keys: ceil(b/8) 8-bit digit passes per half, b = bits of a vertex id;
    # a pass reads every key twice (histogram, scatter) and writes it once: 24 bytes per key
    vb = max(1, int(args.scale))
    passes = 2 * ((vb + 7) // 8)
    pass_bytes = 24.0 * m * passes
    out["sharder"] = {"raw_edges": m, "ms": bms, "first_call_ms": t_build[0], "sort_bytes_16E": 16.0 * m,
                      "frac_of_16E_at_hbm_peak": 16.0 * m / peak / 1e6 / bms,
                      "radix_passes": passes, "radix_pass_bytes": pass_bytes,
                      "frac_of_radix_pass_bytes_at_hbm_peak": pass_bytes / peak / 1e6 / bms,
                      "note": "dedup + in-CSR + degrees + 64 intervals, whole build timed; 16E is the one-pass "
                              "lower bound of a sort, radix_pass_bytes what the LSD passes move (24 B per key "
                              "per pass); the scatter pass is bound by shared-memory bank conflicts"}

    # ---- the vertex-API in-memory program (bit-exact Gauss-Seidel) to the tolerance ----
    s, d = dev_edges(args.scale, args.ef << args.scale, args.seed)
    with gcgpu.Graph.from_edges(s, d, dedup=True, nshards=args.nshards, out_csr=False) as g:
        del s, d
        o = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")
        runs = [g.pagerank(mode=gcgpu.PR_GS_EXACT, max_sweeps=args.max_sweeps, tol=args.tol, out=o)[1]
                for _ in range(2)]
        st = min(runs, key=lambda x: x.device_ms)
        out["gs_exact"] = {"graph": f"rmat{args.scale}_ef{args.ef}_seed{args.seed}", "sweeps_to_tol": st.sweeps,
                           "converged": st.converged, "residual": st.residual, "levels": st.levels,
                           "ms": st.device_ms, "GTEPS": g.num_edges * st.sweeps / st.device_ms / 1e6,
                           "note": "example_apps/pagerank.cpp in-memory program, id-ordered Gauss-Seidel, "
                                   "bit-exact; levels of the u<v in-edge dependency schedule, one launch each "
                                   "per sweep (CUDA graph); time excludes the level schedule's construction"}
        del o

    # ---- connected components (and triangles at scale 20) ----
    cc = {}
    for scale in (24, 20):
        s, d = dev_edges(scale, args.ef << scale, args.seed)
        with gcgpu.Graph.from_edges(s, d, dedup=True, symmetrise=True, out_csr=False) as g:
            del s, d
            V, E = g.num_vertices, g.num_edges
            lab = torch.empty(V, dtype=torch.int32, device="cuda")
            g.connected_components(out=lab)
            ms = min(g.connected_components(out=lab)[1].device_ms for _ in range(3))
            alg = 8.0 * E + 12.0 * V
            row = {"vertices": V, "directed_edges": E, "ms": ms, "GTEPS": E / ms / 1e6,
                   "one_pass_bytes": alg, "one_pass_ms_at_peak": alg / peak / 1e6,
                   "frac_of_one_pass_at_hbm_peak": alg / peak / 1e6 / ms,
                   "note": "sampled scheme: time against one streaming pass over the graph (8E + 12V bytes) "
                           "at the measured HBM peak; most edges are never read"}
            if scale == 20:
                tri, _, _, tst = g.triangle_count(per_rank=False, vertexmap=False)
                tms = min(g.triangle_count(per_rank=False, vertexmap=False)[3].device_ms for _ in range(2))
                row["triangles"] = tri
                row["tc_ms"] = tms
            cc[f"rmat{scale}_sym"] = row
    out["cc"] = cc

    # ---- learned warm start on the headline graph ----
    s, d = dev_edges(args.scale, args.ef << args.scale, args.seed)
    with gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=False) as g, gcgpu.Mlp.load(gw.MODEL_PATH) as m:
        del s, d
        rec = min((gw.evaluate(g, m) for _ in range(2)), key=lambda r: r["ms_warm"])
        out["warm_start"] = {"graph": f"rmat{args.scale}_ef{args.ef}_seed{args.seed}", "model": "gcgpu/warm_start_rmat.npz",
                             "sweeps_plain": rec["sweeps_plain"], "sweeps_warm": rec["sweeps_warm"],
                             "ms_plain": rec["ms_plain"], "ms_warm_total": rec["ms_warm"],
                             "ms_warm_start": rec["ms_warm_start"], "speedup": rec["ms_plain"] / rec["ms_warm"],
                             "l1_between_answers": rec["l1_between"], "tol": 1e-8}

    # ---- batched personalised PageRank ----
    s, d = dev_edges(22, args.ef << 22, args.seed + 6)
    with gcgpu.Graph.from_edges(s, d, dedup=True, out_csr=False) as g:
        del s, d
        n = g.num_vertices
        src = np.random.default_rng(3).integers(0, n, 256).astype(np.uint32)
        g.pagerank(max_sweeps=2)
        mat = torch.empty((n, 256), dtype=torch.float32, device="cuda")
        E22 = g.num_edges
        runs = []
        for _ in range(2):
            wl = np.zeros(2 * 1000, np.uint64)
            pst = g.ppr_batched(src, max_sweeps=1000, tol=1e-8, teleport=0.15, out=mat, work_log=wl)[1]
            runs.append((pst.device_ms, pst.sweeps, wl))
        bms, psweeps, wl = min(runs, key=lambda r: r[0])
        # per sweep E(4 + 4k) + 3 V 4k with k the sources still iterating: the column
        # index once, one contribution per edge and source, three values per vertex and source
        upd, gat = int(wl[2 * psweeps - 2]), int(wl[2 * psweeps - 1])
        ppr_bytes = 4.0 * E22 * psweeps + 4.0 * gat + 12.0 * upd
        vec = torch.empty(n, dtype=torch.float32, device="cuda")
        sample = 32
        sms = sum(g.pagerank(max_sweeps=1000, tol=1e-8, teleport=0.15, source=int(v), out=vec)[1].device_ms
                  for v in src[:sample])
        out["batched_ppr"] = {"graph": "rmat22_ef16", "sources": 256, "ms_batched": bms,
                              "ms_single_source_x256": sms * 256 / sample,
                              "single_source_sample": f"{sample} of the 256 sources timed, scaled by 8",
                              "speedup": sms * 256 / sample / bms, "sweeps": psweeps,
                              "source_sweeps": gat // max(1, E22),
                              "algorithmic_bytes": ppr_bytes,
                              "achieved_gbs": ppr_bytes / bms / 1e6,
                              "frac_of_hbm_peak": ppr_bytes / bms / 1e6 / peak}
        del mat

    # ---- 64 uneven graphs in one persistent launch ----
    rng = np.random.default_rng(5)
    ns = np.exp(rng.uniform(math.log(1e4), math.log(2e6), 64)).astype(int)
    gs = []
    for i, nn in enumerate(ns):
        if i % 2 == 0:
            mm = 8 * int(nn)
            s = torch.empty(mm, dtype=torch.int32, device="cuda")
            d = torch.empty(mm, dtype=torch.int32, device="cuda")
            gcgpu.generate_er(int(nn), mm, 100 + i, s, d)
            gs.append(gcgpu.Graph.from_edges(s, d, num_vertices=int(nn), dedup=True, out_csr=False))
        else:
            sc = max(1, round(math.log2(nn)))
            s, d = dev_edges(sc, 8 << sc, 100 + i)
            gs.append(gcgpu.Graph.from_edges(s, d, num_vertices=1 << sc, dedup=True, out_csr=False))
    seq = 0.0
    for g in gs:
        o = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")
        g.pagerank(max_sweeps=1000, tol=1e-8, out=o)
        seq += g.pagerank(max_sweeps=1000, tol=1e-8, out=o)[1].device_ms
    with gcgpu.Batch(gs) as b:
        hub, run, _ = b.autotune(sweeps=6)
        allr = torch.empty(int(b.offsets[-1]), dtype=torch.float32, device="cuda")
        b.pagerank(max_sweeps=1000, tol=1e-8, out=allr)  # captures the CUDA graph
        best = min((b.pagerank(max_sweeps=1000, tol=1e-8, out=allr) for _ in range(3)), key=lambda x: x[3].device_ms)
        st, gsweeps = best[3], best[1]
        # each graph's own sweeps x (8 E + 16 V), the PageRank bytes per sweep
        mg_bytes = float(sum(int(n) * (8.0 * g.num_edges + 16.0 * g.num_vertices) for n, g in zip(gsweeps, gs)))
        out["batched_graphs"] = {"graphs": 64, "vertices": int(b.offsets[-1]),
                                 "edges": int(sum(g.num_edges for g in gs)), "ms_one_launch": st.device_ms,
                                 "ms_one_solve_per_graph": seq, "speedup": seq / st.device_ms,
                                 "autotuned": {"hub_entries": hub, "queue_run": run}, "cuda_graph": b.config()[2],
                                 "max_sweeps": st.sweeps, "algorithmic_bytes": mg_bytes,
                                 "achieved_gbs": mg_bytes / st.device_ms / 1e6,
                                 "frac_of_hbm_peak": mg_bytes / st.device_ms / 1e6 / peak}
    for g in gs:
        g.free()
    return out


def run_ours(args, rank, world):
    import numpy as np
    import torch
    import torch.distributed as dist
    import gcgpu

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    m = args.ef << args.scale

    # ---- input: seeded R-MAT on the device, sharded on the device ----
    ts = torch.empty(m, dtype=torch.int32, device="cuda")
    td = torch.empty(m, dtype=torch.int32, device="cuda")
    gcgpu.generate_rmat(args.scale, m, 0.57, 0.19, 0.19, seed=args.seed, src=ts, dst=td)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = gcgpu.Graph.from_edges(ts, td, dedup=True, nshards=args.nshards, out_csr=False)
    torch.cuda.synchronize()
    shard_s = time.perf_counter() - t0
    V, E = g.num_vertices, g.num_edges
    g.set_stream(stream.cuda_stream)
    out = torch.empty(V, dtype=torch.float32, device="cuda")

    def solve(time_sweeps=False):
        return g.pagerank(max_sweeps=args.max_sweeps, tol=args.tol, out=out, time_sweeps=time_sweeps)[1]

    for _ in range(args.warmup):
        st = solve()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    # ---- timed region: K solves, inputs resident ----
    stats = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        # the edge kernel's launches are bracketed by CUDA events in the last step
        # only (events between the sweep kernels cost ~2 % of a solve)
        for i in range(args.steps):
            stats.append(solve(time_sweeps=(i == args.steps - 1)))
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    sweeps = [s.sweeps for s in stats]
    value = whole_job_gteps(sum(E * s for s in sweeps), world, ms / 1e3)
    launches = sum(s.kernel_launches for s in stats)
    kern_ms = sum(s.sweep_kernel_ms for s in stats)
    kern_n = sum(s.timed_sweeps for s in stats)
    per_launch_s = kern_ms / kern_n / 1e3
    alg_bytes = 8.0 * E + 16.0 * V
    achieved = alg_bytes / per_launch_s / 1e9
    peak, peak_kind = load_peaks()
    traffic = TRAFFIC_BYTES_PER_EDGE * E if args.scale == 24 else None
    gpu_rank = out.cpu().numpy()

    # ---- e2e: host buffers through the C ABI ----
    hs = torch.empty(m, dtype=torch.int32, pin_memory=True)
    hd = torch.empty(m, dtype=torch.int32, pin_memory=True)
    hs.copy_(ts)
    hd.copy_(td)
    del ts, td
    # the result lands in pinned host memory, as the inputs come from it
    host_rank = torch.zeros(V, dtype=torch.float32, pin_memory=True).numpy()
    e2e_times, e2e_edges = [], 0
    for i in range(args.e2e_warmup + args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with gcgpu.Graph.from_edges(hs, hd, dedup=True, nshards=args.nshards, out_csr=False) as ge:
            _, st = ge.pagerank(max_sweeps=args.max_sweeps, tol=args.tol, out=host_rank)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if i >= args.e2e_warmup:
            e2e_times.append(dt)
            e2e_edges += E * st.sweeps
    e2e_s = max_over_ranks(sum(e2e_times) if e2e_times else float("nan"), world, "cuda")
    e2e_value = whole_job_gteps(e2e_edges, world, e2e_s) if e2e_times else None

    # ---- oracle check and CPU baseline: the oracle on the same graph, host cores ----
    cpu, check = None, None
    if rank == 0 and world == 1 and not (args.no_oracle_check and args.no_cpu_baseline):
        threads = os.cpu_count() or 1
        try:
            check = oracle_check(args.scale, args.ef, args.seed, args.tol, gpu_rank, sweeps[0], threads)
            if check["vertices"] != V or check["edges"] != E:
                raise RuntimeError(f"oracle graph differs: {check['vertices']} x {check['edges']} vs {V} x {E}")
            cpu = {"value": E * check["fp32_sweeps"] / check["fp32_s"] / 1e9, "unit": UNIT, "cores": threads,
                   "kind": "port", "time_to_tol_s": check["fp32_s"], "sweeps": check["fp32_sweeps"],
                   "sample": (f"the whole workload: oracle/oracle.c orc_pagerank_jacobi_mt (the reference's "
                              f"bulk-synchronous PageRank, pagerank_functional.cpp:48-83 with the 0.15 + 0.85 sum "
                              f"apply, restated in C with OpenMP over rows) from the uniform start to residual "
                              f"{args.tol:g} on the same R-MAT scale-{args.scale} graph, {threads} threads; "
                              f"GTEPS = edges x sweeps / time")}
        except Exception as e:  # noqa: BLE001
            check = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
        if args.no_cpu_baseline:
            cpu = None
        if args.no_oracle_check:
            check = None

    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            extras = run_extras(args)
        except Exception as e:  # noqa: BLE001
            extras = {"unavailable": f"{type(e).__name__}: {e}"[:300]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"pagerank_rmat{args.scale}_ef{args.ef}_to_{args.tol:g}",
                       "vertices": V, "edges": E, "raw_edges": m, "nshards": args.nshards,
                       "sweeps_per_step": sweeps[0], "residual": stats[-1].residual,
                       "teleport": 0.15, "damping": 0.85, "init": 1.0,
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "l2": "inputs larger than L2 (col index array alone > 126 MB)",
                       "first_build_ms": shard_s * 1e3,
                       "first_build_note": "the process's first graph build, incl. loading the library's kernels; "
                                           "steady-state sharder time: extras.sharder.ms"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": "k_pr_edges",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": per_launch_s * 1e3,
                         "peak_kind": peak_kind},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * m, "d2h_bytes_per_step": 4 * V,
                    "ms_per_step": e2e_s / max(1, args.e2e_steps) * 1e3},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "oracle_check": check,
            "cpu_baseline": cpu,
            "extras": extras,
        }
        print(json.dumps(line))
    g.free()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gcgpu", choices=["gcgpu", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-sweeps", type=int, default=1000)
    ap.add_argument("--nshards", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-check", action="store_true", help="skip the host oracle's check of the answer")
    ap.add_argument("--no-ref-inmem", action="store_true",
                    help="reference arm: only the default-configuration run (skip the in-memory mode's)")
    ap.add_argument("--no-extras", action="store_true", help="skip the CC / warm-start / batched rows")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
