"""Generates tests/golden/*.npz by running the reference's own compiled apps
(oracle/_ref, built by `make -C oracle ref` from the reference sources) on
seeded synthetic graphs. Run from the repository root where the reference tree
is present:

    make -C oracle lib ref && python tests/golden/make_golden.py

Each case records the generator parameters (so a test can rebuild the exact
input with the numpy restatement in oracle/oracle.py or the library's own
generator), the canonical edge count, and what the reference wrote:
intervals, degrees, decoded shard adjacency, vertex values of PageRank
(vertex API = Gauss-Seidel, functional sync = Jacobi, and a residual-stopped
Jacobi run), connected-component labels and triangle counts. Large arrays are
stored as SHA-256 digests of their little-endian bytes.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
THREADS = int(os.environ.get("GOLDEN_THREADS", "8"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_input(spec):
    kind = spec["kind"]
    if kind == "rmat":
        s, d = O.rmat_numpy(spec["scale"], spec["ef"] << spec["scale"], spec.get("a", 0.57),
                            spec.get("b", 0.19), spec.get("c", 0.19), spec["seed"])
    elif kind == "er":
        s, d = O.er_numpy(spec["n"], spec["m"], spec["seed"])
    elif kind == "explicit":
        s, d = np.array(spec["src"], np.uint32), np.array(spec["dst"], np.uint32)
    else:
        raise ValueError(kind)
    return s, d


def canonical(spec, s, d):
    return O.canonical_edges(s, d, symmetrise=spec.get("sym", False), dedup=True)


def run_case(name, spec, tasks, store_full, merge=False):
    """merge: keep the fields already stored for this case and (re)compute only
    the given tasks."""
    print(f"== {name}", flush=True)
    raw_s, raw_d = make_input(spec)
    s, d = canonical(spec, raw_s, raw_d)
    nv = O.num_vertices(s, d)
    rec = {"spec": json.dumps(spec), "ne": len(s), "nv": nv}
    path = os.path.join(OUT, f"{name}.npz")
    if merge and os.path.exists(path):
        old = dict(np.load(path, allow_pickle=False))
        assert str(old["spec"]) == rec["spec"] and int(old["ne"]) == rec["ne"], "case input changed"
        old.update(rec)
        rec = old
    def put(k, a):
        # tolerance-compared PageRank vectors are always stored in full
        if store_full or k.startswith(("pr_func", "pr_oracle")):
            rec[k] = a
        else:
            rec[k + "_sha"] = sha(a)
    with O.RefWorkdir() as w:
        def fresh(tag):
            p = w.file(f"{tag}.el")
            O.write_edgelist(p, s, d)
            return p

        if "shard" in tasks:
            for P in tasks["shard"]:
                el = fresh(f"sh{P}")
                O.run_ref("pagerank", el, {"niters": 1, "nshards": P}, THREADS)
                iv = O.read_intervals(el, P)
                rec[f"intervals_{P}"] = iv
                rec[f"numvertices_{P}"] = O.read_numvertices(el)
                put(f"degrees_{P}", O.read_degrees(el))
                ss, dd = [], []
                for p in range(len(iv)):
                    a, b = O.decode_shard_adj(f"{el}.edata_azv.{p}_{P}.adj")
                    ss.append(a)
                    dd.append(b)
                rec[f"shard_sizes_{P}"] = np.array([len(x) for x in ss], np.int64)
                put(f"shard_src_{P}", np.concatenate(ss))
                put(f"shard_dst_{P}", np.concatenate(dd))
        if "pr_gs" in tasks:
            for niters, P, budget in tasks["pr_gs"]:
                el = fresh(f"prgs{niters}_{P}_{budget}")
                opts = {"niters": niters, "nshards": P}
                if budget:
                    opts["membudget_mb"] = budget
                O.run_ref("pagerank", el, opts, THREADS)
                put(f"pr_gs_{niters}_{P}_{budget}", O.read_vout(el, np.float32, nv))
                rec[f"pr_gs_{niters}_{P}_{budget}_deltalog"] = np.frombuffer(open(el + ".deltalog", "rb").read(),
                                                                            np.uint8)
        if "pr_edge" in tasks:
            # the edge-value program (pagerank.cpp:73-113): the app takes it when
            # num_vertices * 4 >= membudget; one exec thread keeps the delta sums in
            # vertex order, and shards of <= 1M edges keep each in-edge list in source
            # order (memoryshard.hpp:400-401 decodes larger shards in parallel chunks)
            for niters, P, budget in tasks["pr_edge"]:
                el = fresh(f"pre{niters}_{P}_{budget}")
                out, _ = O.run_ref("pagerank", el, {"niters": niters, "nshards": P, "membudget_mb": budget}, 1)
                assert "in-memory mode" not in out, "the reference took the in-memory program"
                tag = f"pr_edge_{niters}_{P}_{budget}"
                put(tag, O.read_vout(el, np.float32, nv))
                rec[tag + "_deltalog"] = np.frombuffer(open(el + ".deltalog", "rb").read(), np.uint8)
        if "pr_func" in tasks:
            for niters in tasks["pr_func"]:
                el = fresh(f"prf{niters}")
                O.run_ref("pagerank_functional", el, {"niters": niters, "mode": "sync"}, THREADS)
                put(f"pr_func_{niters}", O.read_vout(el, np.float32, nv))
        if "pr_oracle" in tasks:
            for niters, tol in tasks["pr_oracle"]:
                el = fresh(f"pro{niters}")
                out, _ = O.run_ref("pr_functional_oracle", el,
                                   {"niters": niters, "teleport": "const", "tol": tol}, THREADS)
                it = int([ln for ln in out.splitlines() if ln.startswith("iterations")][-1].split()[1])
                res = [float(ln.split()[2]) for ln in out.splitlines() if ln.startswith("residual")]
                tag = f"pr_oracle_{niters}_{tol:g}"
                rec[tag + "_iters"] = it
                rec[tag + "_res"] = np.array(res, np.float64)
                put(tag, O.read_vout(el, np.float32, nv))
        if "cc" in tasks:
            el = fresh("cc")
            O.run_ref("connectedcomponents", el, {}, THREADS)
            lab = O.read_vout(el, np.uint32, nv)
            put("cc", lab)
            rec["cc_ncomp"] = int((lab == np.arange(nv, dtype=np.uint32)).sum())
            # analyze_labels' file, written by the app itself (labelanalysis.hpp:99-176)
            put("cc_components", np.frombuffer(open(el + ".components", "rb").read(), np.uint8))
        if "tc" in tasks:
            P = tasks["tc"]
            el = fresh("tc")
            out, _ = O.run_ref("trianglecounting", el, {"nshards": P}, THREADS)
            line = [ln for ln in out.splitlines() if ln.startswith("Number of triangles")][-1]
            rec["tc_total"] = int(line.split(":")[1].split("(")[0])
            put("tc_per_rank", O.read_vout(el + "_degord", np.uint32, nv))
            put("tc_vertexmap", np.fromfile(el + ".vertexmap", dtype=np.uint32)[:nv])
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in rec.items()})


AGG_N = (1 << 20) + 16
AGG_RANGES = [(0, (1 << 20) + 1), (0, (1 << 20) + 2), (0, AGG_N), (7, (1 << 20) + 8), (5, 6), (0, 1),
              (0, 1000), (3, (1 << 20) + 3)]


def aggregate_values():
    """Seeded uint32 vertex values for the sum_vertices case (small values, so the
    sums stay exact in any order)."""
    return np.random.default_rng(11).integers(0, 1000, AGG_N).astype(np.uint32)


def run_aggregates():
    """sum_vertices (vertex_aggregator.hpp:68-127) over ranges whose last 2^20
    window holds one vertex, computed by the reference's own reader through
    oracle/_ref/aggregate_probe."""
    print("== aggregates", flush=True)
    vals = aggregate_values()
    sums = []
    with O.RefWorkdir() as w:
        base = w.file("agg")
        vals.tofile(base + ".4B.vout")
        with open(base + ".numvertices", "w") as f:
            f.write(f"{AGG_N}\n")
        for a, b in AGG_RANGES:
            out, _ = O.run_probe("sum", base, a, b)
            sums.append(int(re.findall(r"sum (\d+)", out)[-1]))
    np.savez_compressed(os.path.join(OUT, "aggregates.npz"), n=AGG_N, seed=11,
                        ranges=np.array(AGG_RANGES, np.uint64), sums=np.array(sums, np.uint64),
                        values_sha=sha(vals))


CASES = [
    # small, full arrays
    ("rmat_s10_ef16_seed1", {"kind": "rmat", "scale": 10, "ef": 16, "seed": 1},
     {"shard": [1, 4, 7], "pr_gs": [(4, 1, 0), (4, 4, 1), (6, 2, 0)], "pr_func": [4],
      "pr_oracle": [(4, 0.0), (400, 1e-8)], "cc": True, "tc": 2}, True),
    ("er_n3000_m24000_seed3", {"kind": "er", "n": 3000, "m": 24000, "seed": 3},
     {"shard": [3], "pr_gs": [(4, 1, 0)], "pr_func": [4], "cc": True, "tc": 3}, True),
    ("rmat_s12_ef8_sym_seed2", {"kind": "rmat", "scale": 12, "ef": 8, "seed": 2, "sym": True},
     {"shard": [2], "cc": True, "tc": 2, "pr_gs": [(4, 1, 0)]}, True),
    ("handmade_components", {"kind": "explicit",
                             "src": [0, 1, 2, 2, 5, 6, 7, 9, 9, 10, 12, 12, 13, 3, 4, 14, 14, 15, 20, 20, 21],
                             "dst": [1, 2, 0, 3, 6, 7, 5, 10, 11, 11, 13, 14, 14, 4, 3, 15, 16, 16, 21, 22, 22]},
     {"shard": [1, 3], "pr_gs": [(4, 1, 0), (5, 1, 0)], "pr_func": [4], "cc": True, "tc": 2}, True),
    # config 1: PageRank scale 16, 4 iterations (vertex API); CC/TC on the symmetrised graph
    ("rmat_s16_ef16_seed1", {"kind": "rmat", "scale": 16, "ef": 16, "seed": 1},
     {"shard": [1, 8], "pr_gs": [(4, 1, 0)], "pr_func": [4], "pr_oracle": [(4, 0.0)]}, False),
    ("rmat_s16_ef16_sym_seed1", {"kind": "rmat", "scale": 16, "ef": 16, "seed": 1, "sym": True},
     {"cc": True, "tc": 2}, False),
    # the edge-value PageRank program (taken when num_vertices * 4 >= membudget):
    # 1 MB budget, more than 2^18 vertices
    ("er_n300000_m2400000_seed7", {"kind": "er", "n": 300000, "m": 2400000, "seed": 7},
     {"pr_edge": [(5, 4, 1), (2, 4, 1)]}, False),
    ("rmat_s19_ef16_seed3", {"kind": "rmat", "scale": 19, "ef": 16, "seed": 3},
     {"pr_edge": [(4, 12, 1)]}, False),
    # config 3's PageRank program at scale 20: the in-memory vertex program, 4
    # iterations, 20 shards of <= 1M edges
    ("rmat_s20_ef16_seed1", {"kind": "rmat", "scale": 20, "ef": 16, "seed": 1},
     {"pr_gs": [(4, 20, 0)]}, False),
    # config 2: CC and TC at scale 20, symmetrised (digests only)
    ("rmat_s20_ef16_sym_seed2", {"kind": "rmat", "scale": 20, "ef": 16, "seed": 2, "sym": True},
     {"cc": True, "tc": 4}, False),
]

if __name__ == "__main__":
    # python make_golden.py [case ...]            (re)makes the named cases (all by default)
    # python make_golden.py --tasks cc,x case...  recomputes only those tasks, keeping the rest
    if not O.ref_available():
        sys.exit("oracle/_ref is not built: run `make -C oracle lib ref` where the reference tree is present")
    argv = sys.argv[1:]
    only_tasks = None
    if argv[:1] == ["--tasks"]:
        only_tasks = set(argv[1].split(","))
        argv = argv[2:]
    only = set(argv)
    for name, spec, tasks, full in CASES:
        if only and name not in only:
            continue
        if only_tasks is not None:
            tasks = {k: v for k, v in tasks.items() if k in only_tasks}
            if not tasks:
                continue
        run_case(name, spec, tasks, full, merge=only_tasks is not None)
    if not only or "aggregates" in only:
        run_aggregates()
