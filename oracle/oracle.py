"""ORACLE — test infrastructure only.

Python side of the oracle: ctypes wrappers of the plain-C restatement
(oracle/liboracle.so, built from oracle.c), a numpy restatement of the seeded
R-MAT / Erdos-Renyi generators (to check the library's generators
independently), and helpers that run the reference's own compiled apps
(oracle/_ref/, built by oracle/Makefile from the reference sources) and read
their output files. Only tests/, the smoke check and bench.py's CPU-baseline
and reference legs may use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "lib"], check=True, capture_output=True)
        _lib = C.CDLL(LIB_PATH)
        _vp, _u32, _u64, _i, _d, _f = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double, C.c_float
        for name, res, args in [
            ("orc_canonical_edges", _u64, [_vp, _vp, _u64, _i, _i, _vp, _vp]),
            ("orc_build_csr", None, [_u32, _vp, _vp, _u64, _i, _vp, _vp]),
            ("orc_intervals", _u32, [_vp, _u32, _u32, _vp]),
            ("orc_auto_nshards", _u32, [_u64, _u32, _u32]),
            ("orc_pagerank_gs_inmem", None, [_u32, _vp, _vp, _vp, _i, _vp]),
            ("orc_pagerank_gs_edge", None, [_u32, _vp, _vp, _vp, _i, _vp, _vp]),
            ("orc_pagerank_gs_track", _i, [_u32, _vp, _vp, _vp, _i, _i, _d, _vp, _vp, _vp]),
            ("orc_pagerank_jacobi", _i, [_u32, _vp, _vp, _vp, _d, _d, _f, _i, _d, _vp, _vp]),
            ("orc_pagerank_jacobi_f64", _i, [_u32, _vp, _vp, _vp, _d, _d, _d, _i, _d, _vp]),
            ("orc_cc", _i, [_u32, _vp, _vp, _vp, _vp, _vp]),
            ("orc_tc", _u64, [_u32, _vp, _vp, _vp, _vp, _vp, _vp]),
            ("orc_ppr", _i, [_u32, _vp, _vp, _vp, _vp, _u32, _d, _i, _d, _vp]),
            ("orc_write_edgelist", _i, [C.c_char_p, _vp, _vp, _u64]),
            ("orc_rmat_edges", None, [_u32, _u64, _d, _d, _d, _u64, _vp, _vp]),
            ("orc_in_csr_mt", _u64, [_vp, _vp, _u64, _u32, _vp, _vp, _vp, _vp]),
            ("orc_pagerank_jacobi_mt", _i, [_u32, _vp, _vp, _vp, _d, _d, _f, _i, _d, _vp, _vp]),
            ("orc_pagerank_jacobi_f64_mt", _i, [_u32, _vp, _vp, _vp, _d, _d, _d, _vp, _i, _d, _vp, _vp]),
        ]:
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


# ---- graph construction --------------------------------------------------

def canonical_edges(src, dst, symmetrise=False, dedup=True):
    src, dst = _u32(src), _u32(dst)
    m = src.shape[0]
    cap = 2 * m if symmetrise else m
    os_, od = np.zeros(max(cap, 1), np.uint32), np.zeros(max(cap, 1), np.uint32)
    n = lib().orc_canonical_edges(_p(src), _p(dst), m, int(symmetrise), int(dedup), _p(os_), _p(od))
    return os_[:n].copy(), od[:n].copy()


def num_vertices(src, dst):
    """max id + 1 over non-self-loop edges (sharder.hpp:440-445, :925); 1 if none."""
    keep = src != dst
    if not keep.any():
        return 1
    return int(max(src[keep].max(), dst[keep].max())) + 1


def csr(nv, src, dst, by_dst):
    src, dst = _u32(src), _u32(dst)
    rp = np.zeros(nv + 1, np.uint32)
    col = np.zeros(max(1, src.shape[0]), np.uint32)
    lib().orc_build_csr(nv, _p(src), _p(dst), src.shape[0], int(by_dst), _p(rp), _p(col))
    return rp, col[: src.shape[0]]


class OracleGraph:
    """Canonical graph + both CSRs, built by the oracle."""

    @classmethod
    def in_csr_only(cls, src, dst):
        """The in-CSR and out-degrees of the canonical (deduplicated) directed
        graph, built on all host threads: for full-size PageRank checks. The
        canonical edge arrays and the out-CSR are not kept."""
        src, dst = _u32(src), _u32(dst)
        m = src.shape[0]
        cap = int(max(src.max(initial=0), dst.max(initial=0))) + 1
        g = cls.__new__(cls)
        rp = np.zeros(cap + 1, np.uint32)
        col = np.zeros(max(1, m), np.uint32)
        od = np.zeros(cap, np.uint32)
        nv = C.c_uint32(0)
        e = lib().orc_in_csr_mt(_p(src), _p(dst), m, cap, C.addressof(nv), _p(rp), _p(col), _p(od))
        g.nv = int(nv.value)
        g.in_rowptr = rp[: g.nv + 1].copy()
        g.in_col = col[:e]
        g.outdeg = od[: g.nv].copy()
        g.indeg = np.diff(g.in_rowptr).astype(np.uint32)
        g.src = g.dst = g.out_rowptr = g.out_col = None
        g._ne = int(e)
        return g

    def __init__(self, src, dst, symmetrise=False, dedup=True, nv=None, out_csr=True):
        s, d = canonical_edges(src, dst, symmetrise, dedup)
        self.src, self.dst = s, d
        self.nv = nv if nv is not None else num_vertices(s, d)
        self.in_rowptr, self.in_col = csr(self.nv, s, d, True)
        self.indeg = np.diff(self.in_rowptr).astype(np.uint32)
        if out_csr:
            self.out_rowptr, self.out_col = csr(self.nv, s, d, False)
            self.outdeg = np.diff(self.out_rowptr).astype(np.uint32)
        else:  # full-size PageRank checks need only the in-CSR and out-degrees
            self.out_rowptr = self.out_col = None
            self.outdeg = np.bincount(s, minlength=self.nv).astype(np.uint32)

    @property
    def ne(self):
        return self._ne if self.src is None else int(self.src.shape[0])

    def intervals(self, nshards):
        out = np.zeros(max(1, nshards), np.uint32)
        n = lib().orc_intervals(_p(self.in_rowptr), self.nv, nshards, _p(out))
        return out[:n].copy()

    def degrees(self):
        return np.stack([self.indeg.astype(np.int32), self.outdeg.astype(np.int32)], axis=1)

    def pagerank_gs_inmem(self, niters):
        out = np.zeros(self.nv, np.float32)
        lib().orc_pagerank_gs_inmem(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg), niters, _p(out))
        return out

    def pagerank_gs_edge(self, niters):
        """Edge-value vertex program (pagerank.cpp:73-113): (values, delta per iteration)."""
        out = np.zeros(self.nv, np.float32)
        log = np.zeros(max(1, niters), np.float64)
        lib().orc_pagerank_gs_edge(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg), niters, _p(out),
                                   _p(log))
        return out, log[:niters].copy()

    def pagerank_gs_track(self, edge, max_sweeps, tol=0.0):
        """Vertex-API program with per-sweep tracking: (values, sweeps, delta log, residual log)."""
        out = np.zeros(self.nv, np.float32)
        dl = np.zeros(max(1, max_sweeps), np.float64)
        rl = np.zeros(max(1, max_sweeps), np.float64)
        n = lib().orc_pagerank_gs_track(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg), int(edge),
                                        max_sweeps, tol, _p(out), _p(dl), _p(rl))
        return out, n, dl[:n].copy(), rl[:n].copy()

    def pagerank_jacobi(self, teleport=0.15, damping=0.85, init=1.0, max_sweeps=3, tol=0.0):
        out = np.zeros(self.nv, np.float32)
        log = np.zeros(max(1, max_sweeps), np.float64)
        n = lib().orc_pagerank_jacobi(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg),
                                      teleport, damping, init, max_sweeps, tol, _p(out), _p(log))
        return out, n, log[:n].copy()

    def pagerank_jacobi_f64(self, teleport=0.15, damping=0.85, init=1.0, max_sweeps=3, tol=0.0):
        out = np.zeros(self.nv, np.float64)
        n = lib().orc_pagerank_jacobi_f64(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg),
                                          teleport, damping, init, max_sweeps, tol, _p(out))
        return out, n

    def pagerank_jacobi_mt(self, teleport=0.15, damping=0.85, init=1.0, max_sweeps=3, tol=0.0):
        """pagerank_jacobi on all host threads (bit-identical ranks)."""
        out = np.zeros(self.nv, np.float32)
        log = np.zeros(max(1, max_sweeps), np.float64)
        n = lib().orc_pagerank_jacobi_mt(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg),
                                         teleport, damping, init, max_sweeps, tol, _p(out), _p(log))
        return out, n, log[:n].copy()

    def pagerank_jacobi_f64_mt(self, teleport=0.15, damping=0.85, init=1.0, max_sweeps=3, tol=0.0,
                               init_vec=None):
        """pagerank_jacobi_f64 on all host threads; returns (ranks, sweeps, residual log)."""
        out = np.zeros(self.nv, np.float64)
        log = np.zeros(max(1, max_sweeps), np.float64)
        iv = None if init_vec is None else np.ascontiguousarray(init_vec, np.float64)
        n = lib().orc_pagerank_jacobi_f64_mt(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg),
                                             teleport, damping, init, _p(iv), max_sweeps, tol, _p(out), _p(log))
        return out, n, log[:n].copy()

    def cc(self):
        out = np.zeros(self.nv, np.uint32)
        n = lib().orc_cc(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.out_rowptr), _p(self.out_col),
                         _p(out))
        return out, n

    def tc(self):
        per = np.zeros(self.nv, np.uint32)
        vm = np.zeros(self.nv, np.uint32)
        t = lib().orc_tc(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.out_rowptr), _p(self.out_col),
                         _p(per), _p(vm))
        return int(t), per, vm

    def ppr(self, sources, damping=0.85, max_sweeps=100, tol=1e-8):
        sources = _u32(sources)
        k = sources.shape[0]
        out = np.zeros(self.nv * k, np.float32)
        n = lib().orc_ppr(self.nv, _p(self.in_rowptr), _p(self.in_col), _p(self.outdeg), _p(sources), k,
                          damping, max_sweeps, tol, _p(out))
        return out.reshape(self.nv, k), n


def auto_nshards(nedges, esize=4, membudget_mb=800):
    return lib().orc_auto_nshards(nedges, esize, membudget_mb)


# ---- generator restatement (numpy) ---------------------------------------

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def seed_key(seed):
    return _mix64(np.uint64(seed) ^ np.uint64(0x6A09E667F3BCC909))


def rmat_numpy(scale, m, a=0.57, b=0.19, c=0.19, seed=1):
    """Restatement of gcg_rmat_edge (csrc/gcg_rng.h) in numpy."""
    two32 = 4294967296.0
    ta, tab, tabc = (np.uint64(int(a * two32)), np.uint64(int((a + b) * two32)),
                     np.uint64(int((a + b + c) * two32)))
    key = seed_key(seed)
    i = np.arange(m, dtype=np.uint64)
    ndraw = np.uint64((scale + 1) // 2)
    s = np.zeros(m, np.uint64)
    d = np.zeros(m, np.uint64)
    w = None
    with np.errstate(over="ignore"):
        for lvl in range(scale):
            if lvl % 2 == 0:
                w = _mix64(key + (i * ndraw + np.uint64(lvl // 2 + 1)) * _GOLDEN)
            u = (w & np.uint64(0xFFFFFFFF)) if lvl % 2 else (w >> np.uint64(32))
            q = (u >= ta).astype(np.uint64) + (u >= tab).astype(np.uint64) + (u >= tabc).astype(np.uint64)
            s = (s << np.uint64(1)) | (q >> np.uint64(1))
            d = (d << np.uint64(1)) | (q & np.uint64(1))
    return s.astype(np.uint32), d.astype(np.uint32)


def rmat_edges(scale, m, a=0.57, b=0.19, c=0.19, seed=1):
    """The same generator as rmat_numpy, restated in C (oracle.c) on all host
    threads: for full-size inputs."""
    s = np.empty(m, np.uint32)
    d = np.empty(m, np.uint32)
    lib().orc_rmat_edges(scale, m, a, b, c, seed, _p(s), _p(d))
    return s, d


def er_numpy(n, m, seed=1):
    key = seed_key(seed)
    i = np.arange(m, dtype=np.uint64)
    with np.errstate(over="ignore"):
        w = _mix64(key + (i + np.uint64(1)) * _GOLDEN)
    s = ((w >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)
    d = ((w & np.uint64(0xFFFFFFFF)) * np.uint64(n)) >> np.uint64(32)
    return s.astype(np.uint32), d.astype(np.uint32)


# ---- the reference's own apps --------------------------------------------

REF_APPS = ["pagerank", "pagerank_functional", "connectedcomponents", "trianglecounting",
            "basic_smoketest", "bulksync_functional_test", "pr_functional_oracle", "aggregate_probe"]


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, a)) for a in REF_APPS) and \
        os.path.exists(os.path.join(REF_DIR, "conf", "graphchi.cnf"))


def write_edgelist(path, src, dst):
    """Whitespace edge list "src dst" per line, the input of convert_edgelist."""
    s, d = _u32(src), _u32(dst)
    if lib().orc_write_edgelist(os.fsencode(path), _p(s), _p(d), s.shape[0]) != 0:
        raise OSError(f"could not write {path}")


def run_ref(app, edgelist, opts=None, threads=None, timeout=3600):
    """Runs oracle/_ref/<app> file=<edgelist> filetype=edgelist <opts>.
    Returns (stdout, wall seconds). Outputs land next to the edge list."""
    args = [os.path.join(REF_DIR, app), "file", edgelist, "filetype", "edgelist"]
    for k, v in (opts or {}).items():
        args += [str(k), str(v)]
    if threads:
        args += ["execthreads", str(threads), "loadthreads", str(threads)]
    env = dict(os.environ, GRAPHCHI_ROOT=REF_DIR)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    t0 = time.perf_counter()
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout,
                       cwd=os.path.dirname(os.path.abspath(edgelist)))
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{app} failed ({r.returncode}): {r.stderr[-2000:]}{r.stdout[-2000:]}")
    return r.stdout + r.stderr, dt


def run_probe(*args, timeout=600):
    """Runs oracle/_ref/aggregate_probe (the reference's sum_vertices /
    analyze_labels on a vertex-value file). Returns (stdout, wall seconds)."""
    cmd = [os.path.join(REF_DIR, "aggregate_probe")] + [str(a) for a in args]
    env = dict(os.environ, GRAPHCHI_ROOT=REF_DIR)
    t0 = time.perf_counter()
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"aggregate_probe failed ({r.returncode}): {r.stderr[-2000:]}{r.stdout[-2000:]}")
    return r.stdout + r.stderr, time.perf_counter() - t0


def ref_runtime(output):
    """The engine's own 'runtime' metric (seconds) from a metrics report."""
    m = re.findall(r"runtime:\s*([0-9.eE+-]+)\s*s", output)
    if not m:
        m = re.findall(r"runtime\s*[:=]\s*([0-9.eE+-]+)", output)
    return float(m[-1]) if m else None


def read_vout(base, dtype, n=None):
    a = np.fromfile(f"{base}.{np.dtype(dtype).itemsize}B.vout", dtype=dtype)
    return a if n is None else a[:n]


def read_intervals(base, nshards):
    with open(f"{base}.{nshards}.intervals") as f:
        return np.array([int(x) for x in f.read().split()], dtype=np.uint32)


def read_numvertices(base):
    with open(f"{base}.numvertices") as f:
        return int(f.read().split()[0])


def read_degrees(base):
    return np.fromfile(f"{base}_degs.bin", dtype=np.int32).reshape(-1, 2)


def decode_shard_adj(path):
    """Decodes a shard adjacency file (format written by sharder::finish_shard,
    src/preprocessing/sharder.hpp:774-818): per source vertex a count byte
    (or 0xff + uint32 count) followed by the uint32 destinations; a zero count
    byte is followed by the number of further vertices without edges.
    Returns (src, dst) arrays in file order."""
    data = open(path, "rb").read()
    pos, vid = 0, 0
    srcs, dsts = [], []
    n = len(data)
    while pos < n:
        c = data[pos]
        pos += 1
        if c == 0:
            nz = data[pos]
            pos += 1
            vid += nz + 1
            continue
        if c == 0xFF:
            cnt = int.from_bytes(data[pos:pos + 4], "little")
            pos += 4
        else:
            cnt = c
        d = np.frombuffer(data, dtype=np.uint32, count=cnt, offset=pos)
        pos += 4 * cnt
        srcs.append(np.full(cnt, vid, np.uint32))
        dsts.append(d.copy())
        vid += 1
    if not srcs:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    return np.concatenate(srcs), np.concatenate(dsts)


class RefWorkdir:
    """Scratch directory for one reference run (the apps write next to the input)."""

    def __init__(self, prefix="gcg_ref_"):
        self.path = tempfile.mkdtemp(prefix=prefix)

    def file(self, name):
        return os.path.join(self.path, name)

    def close(self):
        shutil.rmtree(self.path, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
