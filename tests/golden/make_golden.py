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


def run_case(name, spec, tasks, store_full):
    print(f"== {name}", flush=True)
    raw_s, raw_d = make_input(spec)
    s, d = canonical(spec, raw_s, raw_d)
    nv = O.num_vertices(s, d)
    rec = {"spec": json.dumps(spec), "ne": len(s), "nv": nv}
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
        if "tc" in tasks:
            P = tasks["tc"]
            el = fresh("tc")
            out, _ = O.run_ref("trianglecounting", el, {"nshards": P}, THREADS)
            line = [ln for ln in out.splitlines() if ln.startswith("Number of triangles")][-1]
            rec["tc_total"] = int(line.split(":")[1].split("(")[0])
            put("tc_per_rank", O.read_vout(el + "_degord", np.uint32, nv))
            put("tc_vertexmap", np.fromfile(el + ".vertexmap", dtype=np.uint32)[:nv])
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **{k: np.asarray(v) for k, v in rec.items()})


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
    # config 2: CC and TC at scale 20, symmetrised (digests only)
    ("rmat_s20_ef16_sym_seed2", {"kind": "rmat", "scale": 20, "ef": 16, "seed": 2, "sym": True},
     {"cc": True, "tc": 4}, False),
]

if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref is not built: run `make -C oracle lib ref` where the reference tree is present")
    only = set(sys.argv[1:])
    for name, spec, tasks, full in CASES:
        if only and name not in only:
            continue
        run_case(name, spec, tasks, full)
