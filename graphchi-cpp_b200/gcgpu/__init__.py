"""ctypes binding of libgcgpu, the C ABI declared in include/gcgpu.h.

This is plumbing for Python callers (tests, bench): every call goes straight to
the CUDA library. There is no CPU fallback: if ``lib/libgcgpu.so`` has not been
built, importing this package raises ImportError.

Arrays may be numpy arrays (host memory) or CUDA torch tensors (device memory);
the library uses device memory in place and stages host memory itself.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libgcgpu.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libgcgpu.so not found at {LIB_PATH}: build it with `make -C graphchi-cpp_b200` "
        "(or __graft_entry__.build()); there is no CPU fallback")

_lib = C.CDLL(LIB_PATH)

GCG_OK = 0
STATUS_NAMES = {0: "GCG_OK", -1: "GCG_ERR_INVALID", -2: "GCG_ERR_CUDA", -3: "GCG_ERR_NOMEM",
                -4: "GCG_ERR_IO", -5: "GCG_ERR_FORMAT", -6: "GCG_ERR_UNSUPPORTED",
                -7: "GCG_ERR_TIMEOUT"}

BUILD_DEDUP = 0x1
BUILD_SYMMETRISE = 0x2
BUILD_NO_OUT_CSR = 0x4
CSR_IN = 0
CSR_OUT = 1
PR_JACOBI = 0
PR_GS_EXACT = 1
PR_DELTA = 2
PR_GS_EDGE = 3
PR_TIME_SWEEPS = 0x1
BATCH_ONE_HUB = 0x1

# Every symbol include/gcgpu.h declares (checked by the CPU test suite).
EXPORTED = [
    "gcg_graph_from_edges", "gcg_graph_from_edgelist_file", "gcg_parse_edgelist_file",
    "gcg_graph_free", "gcg_graph_set_stream", "gcg_graph_get_info", "gcg_graph_intervals",
    "gcg_graph_degrees", "gcg_graph_csr", "gcg_graph_write_metadata", "gcg_write_vout",
    "gcg_pr_params_default", "gcg_pagerank", "gcg_connected_components", "gcg_triangle_count",
    "gcg_generate_rmat", "gcg_generate_er", "gcg_last_error", "gcg_version",
    "gcg_pagerank_csr_noalloc", "gcg_ppr_batched",
    "gcg_batch_create", "gcg_batch_create_ex", "gcg_batch_vertex_offsets", "gcg_batch_set_stream", "gcg_batch_pagerank", "gcg_batch_free",
    "gcg_batch_autotune", "gcg_batch_get_config", "gcg_batch_set_config",
    "gcg_pagerank_set_config", "gcg_pagerank_get_config", "gcg_pagerank_autotune",
    "gcg_pagerank_set_tiers", "gcg_pagerank_get_tiers",
    "gcg_connected_components_ex", "gcg_graph_get_device_view", "gcg_graph_add_edges", "gcg_graph_delete_edges",
    "gcg_mlp_create", "gcg_mlp_free", "gcg_mlp_get", "gcg_mlp_set", "gcg_mlp_fit_normalisation",
    "gcg_warm_features", "gcg_mlp_forward", "gcg_mlp_gradient", "gcg_mlp_train_params_default", "gcg_mlp_train",
    "gcg_warm_start_rank", "gcg_cached_memory", "gcg_release_cached_memory",
]
MLP_IN = 8
MLP_HIDDEN = 64
MLP_NPARAMS = 64 * 8 + 64 + 64 * 64 + 64 + 64 + 1
PR_TEST_BARRIER_TIMEOUT = 0x2
NOALLOC_MAX_VERTICES = 1 << 20


class GcgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GraphInfo(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("nshards", C.c_uint32), ("num_edges", C.c_uint64),
                ("has_out_csr", C.c_uint32), ("reserved", C.c_uint32)]


class PrParams(C.Structure):
    _fields_ = [("mode", C.c_int), ("max_sweeps", C.c_int), ("teleport", C.c_double),
                ("damping", C.c_double), ("tol", C.c_double), ("init", C.c_float),
                ("flags", C.c_uint32), ("init_rank", C.c_void_p), ("residuals", C.c_void_p),
                ("source", C.c_uint32), ("reserved2", C.c_uint32), ("delta_log", C.c_void_p),
                ("work_log", C.c_void_p), ("delta_threshold", C.c_double)]


NO_SOURCE = 0xFFFFFFFF


class PrStats(C.Structure):
    _fields_ = [("sweeps", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("device_ms", C.c_double), ("sweep_kernel_ms", C.c_double), ("timed_sweeps", C.c_int),
                ("kernel_launches", C.c_int), ("levels", C.c_int)]


class MlpTrainParams(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64)]


class CcStats(C.Structure):
    _fields_ = [("passes", C.c_int), ("ncomponents", C.c_uint32), ("device_ms", C.c_double)]


class CcParams(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("scheduler", C.c_int), ("max_iterations", C.c_int),
                ("reserved", C.c_uint32), ("frontier_log", C.c_void_p)]


CC_UNION_FIND = 0
CC_LABEL_PROPAGATION = 1


class TcStats(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("oriented_edges", C.c_uint64), ("device_ms", C.c_double)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_vp = C.c_void_p
_u32, _u64, _i = C.c_uint32, C.c_uint64, C.c_int
_graph_from_edges = _sig("gcg_graph_from_edges", _i, _vp, _vp, _u64, _u32, _u32, _u32, C.POINTER(_vp))
_graph_from_file = _sig("gcg_graph_from_edgelist_file", _i, C.c_char_p, _u32, _u32, C.POINTER(_vp))
_parse_file = _sig("gcg_parse_edgelist_file", _i, C.c_char_p, _vp, _vp, _u64, C.POINTER(_u64))
_graph_free = _sig("gcg_graph_free", _i, _vp)
_graph_add = _sig("gcg_graph_add_edges", _i, _vp, _vp, _vp, _u64)
_graph_del = _sig("gcg_graph_delete_edges", _i, _vp, _vp, _vp, _u64)
_graph_set_stream = _sig("gcg_graph_set_stream", _i, _vp, _vp)
_graph_info = _sig("gcg_graph_get_info", _i, _vp, C.POINTER(GraphInfo))
_graph_intervals = _sig("gcg_graph_intervals", _i, _vp, _vp)
_graph_degrees = _sig("gcg_graph_degrees", _i, _vp, _vp)
_graph_csr = _sig("gcg_graph_csr", _i, _vp, _i, _vp, _vp)
_write_meta = _sig("gcg_graph_write_metadata", _i, _vp, C.c_char_p)
_write_vout = _sig("gcg_write_vout", _i, C.c_char_p, _vp, _u32, _u32)
_pr_default = _sig("gcg_pr_params_default", None, C.POINTER(PrParams))
_pagerank = _sig("gcg_pagerank", _i, _vp, C.POINTER(PrParams), _vp, C.POINTER(PrStats))
_cc = _sig("gcg_connected_components", _i, _vp, _vp, C.POINTER(CcStats))
_cc_ex = _sig("gcg_connected_components_ex", _i, _vp, C.POINTER(CcParams), _vp, C.POINTER(CcStats))
_tc = _sig("gcg_triangle_count", _i, _vp, _vp, _vp, _vp, C.POINTER(TcStats))
_gen_rmat = _sig("gcg_generate_rmat", _i, _u32, _u64, C.c_double, C.c_double, C.c_double, _u64, _vp, _vp)
_gen_er = _sig("gcg_generate_er", _i, _u32, _u64, _u64, _vp, _vp)
_pr_noalloc = _sig("gcg_pagerank_csr_noalloc", _i, _vp, _vp, _vp, _u32, C.POINTER(PrParams), _vp, _vp,
                   C.POINTER(PrStats))
_pr_set_config = _sig("gcg_pagerank_set_config", _i, _vp, _u32, _u32)
_pr_get_config = _sig("gcg_pagerank_get_config", _i, _vp, C.POINTER(_u32), C.POINTER(_u32))
_pr_set_tiers = _sig("gcg_pagerank_set_tiers", _i, _vp, _u32)
_pr_get_tiers = _sig("gcg_pagerank_get_tiers", _i, _vp, C.POINTER(_u32))
_pr_autotune = _sig("gcg_pagerank_autotune", _i, _vp, _i, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(C.c_double))
_ppr = _sig("gcg_ppr_batched", _i, _vp, _vp, _u32, C.POINTER(PrParams), _vp, C.POINTER(PrStats))
_batch_create = _sig("gcg_batch_create_ex", _i, C.POINTER(_vp), _u32, _u32, C.POINTER(_vp))
_batch_offsets = _sig("gcg_batch_vertex_offsets", _i, _vp, _vp)
_batch_set_stream = _sig("gcg_batch_set_stream", _i, _vp, _vp)
_batch_pagerank = _sig("gcg_batch_pagerank", _i, _vp, C.POINTER(PrParams), _vp, _vp, _vp, C.POINTER(PrStats))
_batch_free = _sig("gcg_batch_free", _i, _vp)
_batch_autotune = _sig("gcg_batch_autotune", _i, _vp, _i, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(C.c_double))
_batch_set_config = _sig("gcg_batch_set_config", _i, _vp, _u32, _u32)
_batch_get_config = _sig("gcg_batch_get_config", _i, _vp, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_i))
_mlp_create = _sig("gcg_mlp_create", _i, _u64, C.POINTER(_vp))
_mlp_free = _sig("gcg_mlp_free", _i, _vp)
_mlp_get = _sig("gcg_mlp_get", _i, _vp, _vp, _vp)
_mlp_set = _sig("gcg_mlp_set", _i, _vp, _vp, _vp)
_mlp_fit_norm = _sig("gcg_mlp_fit_normalisation", _i, _vp, _vp, _u64)
_warm_features = _sig("gcg_warm_features", _i, _vp, _vp)
_mlp_forward = _sig("gcg_mlp_forward", _i, _vp, _vp, _u64, _vp)
_mlp_gradient = _sig("gcg_mlp_gradient", _i, _vp, _vp, _vp, _u64, _vp, C.POINTER(C.c_double))
_mlp_train_default = _sig("gcg_mlp_train_params_default", None, C.POINTER(MlpTrainParams))
_mlp_train = _sig("gcg_mlp_train", _i, _vp, _vp, _vp, _u64, C.POINTER(MlpTrainParams), _vp)
_warm_start = _sig("gcg_warm_start_rank", _i, _vp, _vp, C.c_double, C.c_double, _vp, C.POINTER(C.c_double))
_last_error = _sig("gcg_last_error", C.c_char_p)
_version = _sig("gcg_version", C.c_char_p)
_cached_memory = _sig("gcg_cached_memory", _i, C.POINTER(_u64), C.POINTER(_u64))
_release_cached = _sig("gcg_release_cached_memory", _i, C.POINTER(_u64))


def last_error() -> str:
    return _last_error().decode()


def version() -> str:
    return _version().decode()


def cached_memory():
    """Idle bytes the library's block cache holds: (device, pinned host)."""
    d, h = _u64(0), _u64(0)
    check(_cached_memory(C.byref(d), C.byref(h)))
    return d.value, h.value


def release_cached_memory() -> int:
    """Returns every idle cached block to the driver; gives the bytes released."""
    b = _u64(0)
    check(_release_cached(C.byref(b)))
    return b.value


def check(status: int) -> None:
    if status != GCG_OK:
        raise GcgError(status, last_error())


def ptr(a):
    """Address of a numpy array (host) or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be contiguous"
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous(), "tensor must be contiguous"
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _u32_host(a):
    if isinstance(a, np.ndarray):
        return np.ascontiguousarray(a, dtype=np.uint32)
    return a


class Graph:
    """Device-resident graph built by the device sharder (gcg_graph_from_edges)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_edges(cls, src, dst, num_vertices=0, dedup=False, symmetrise=False, nshards=1,
                   out_csr=True) -> "Graph":
        src, dst = _u32_host(src), _u32_host(dst)
        m = int(src.shape[0])
        flags = (BUILD_DEDUP if dedup else 0) | (BUILD_SYMMETRISE if symmetrise else 0) | \
                (0 if out_csr else BUILD_NO_OUT_CSR)
        h = _vp()
        check(_graph_from_edges(ptr(src), ptr(dst), m, num_vertices, flags, nshards, C.byref(h)))
        return cls(h)

    @classmethod
    def from_edgelist_file(cls, path, dedup=False, symmetrise=False, nshards=1, out_csr=True) -> "Graph":
        flags = (BUILD_DEDUP if dedup else 0) | (BUILD_SYMMETRISE if symmetrise else 0) | \
                (0 if out_csr else BUILD_NO_OUT_CSR)
        h = _vp()
        check(_graph_from_file(os.fsencode(path), flags, nshards, C.byref(h)))
        return cls(h)

    def free(self):
        if self._h:
            _graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int):
        check(_graph_set_stream(self._h, stream_ptr))

    def add_edges(self, src, dst):
        """gcg_graph_add_edges: the graph becomes its edges plus these (rebuilt on the device)."""
        src, dst = _u32_host(src), _u32_host(dst)
        check(_graph_add(self._h, ptr(src), ptr(dst), int(src.shape[0])))

    def delete_edges(self, src, dst):
        """gcg_graph_delete_edges: removes every copy of each listed edge."""
        src, dst = _u32_host(src), _u32_host(dst)
        check(_graph_del(self._h, ptr(src), ptr(dst), int(src.shape[0])))

    def info(self) -> GraphInfo:
        i = GraphInfo()
        check(_graph_info(self._h, C.byref(i)))
        return i

    @property
    def num_vertices(self) -> int:
        return self.info().num_vertices

    @property
    def num_edges(self) -> int:
        return self.info().num_edges

    def intervals(self) -> np.ndarray:
        out = np.zeros(self.info().nshards, dtype=np.uint32)
        check(_graph_intervals(self._h, ptr(out)))
        return out

    def degrees(self) -> np.ndarray:
        """(V, 2) int32 array of (indegree, outdegree), the _degs.bin layout."""
        out = np.zeros((self.num_vertices, 2), dtype=np.int32)
        check(_graph_degrees(self._h, ptr(out)))
        return out

    def csr(self, which=CSR_IN):
        i = self.info()
        rp = np.zeros(i.num_vertices + 1, dtype=np.uint32)
        col = np.zeros(max(1, i.num_edges), dtype=np.uint32)
        check(_graph_csr(self._h, which, ptr(rp), ptr(col)))
        return rp, col[: i.num_edges]

    def write_metadata(self, base: str):
        check(_write_meta(self._h, os.fsencode(base)))

    def pagerank(self, mode=PR_JACOBI, max_sweeps=3, teleport=0.15, damping=0.85, tol=0.0, init=1.0,
                 init_rank=None, out=None, residuals=None, time_sweeps=False, source=None, delta_log=None,
                 work_log=None, delta_threshold=0.0):
        """Returns (ranks, PrStats). out/init_rank/residuals/delta_log/work_log: numpy or device tensors."""
        p = PrParams()
        _pr_default(C.byref(p))
        p.mode, p.max_sweeps, p.teleport, p.damping, p.tol, p.init = (
            mode, max_sweeps, teleport, damping, tol, init)
        p.delta_threshold = delta_threshold
        if delta_log is not None:
            p.delta_log = ptr(delta_log)
        if work_log is not None:
            p.work_log = ptr(work_log)
        p.flags = PR_TIME_SWEEPS if time_sweeps else 0
        p.source = NO_SOURCE if source is None else int(source)
        if init_rank is not None:
            init_rank = init_rank if not isinstance(init_rank, np.ndarray) else \
                np.ascontiguousarray(init_rank, dtype=np.float32)
            p.init_rank = ptr(init_rank)
        if residuals is not None:
            p.residuals = ptr(residuals)
        if out is None:
            out = np.zeros(self.num_vertices, dtype=np.float32)
        st = PrStats()
        check(_pagerank(self._h, C.byref(p), ptr(out), C.byref(st)))
        return out, st

    def pagerank_config(self, hub_entries=None, chunk_run=None):
        """Sets (when given) and returns the edge kernel's (hub entries, chunk run)."""
        if hub_entries is not None or chunk_run is not None:
            h0, r0 = self.pagerank_config()
            check(_pr_set_config(self._h, h0 if hub_entries is None else hub_entries,
                                 r0 if chunk_run is None else chunk_run))
        h, r = _u32(0), _u32(0)
        check(_pr_get_config(self._h, C.byref(h), C.byref(r)))
        return h.value, r.value

    def pagerank_tiers(self, tiers=None):
        """Sets (when given) and returns the number of source tiers of the edge phase."""
        if tiers is not None:
            check(_pr_set_tiers(self._h, int(tiers)))
        t = _u32(0)
        check(_pr_get_tiers(self._h, C.byref(t)))
        return t.value

    def pagerank_autotune(self, sweeps=8):
        """Times the edge kernel's candidate configurations; returns (hub entries, chunk run, ms per sweep)."""
        h, r, ms = _u32(0), _u32(0), C.c_double(0.0)
        check(_pr_autotune(self._h, sweeps, C.byref(h), C.byref(r), C.byref(ms)))
        return h.value, r.value, ms.value

    def ppr_batched(self, sources, max_sweeps=100, teleport=0.15, damping=0.85, tol=0.0, out=None,
                    residuals=None, time_sweeps=False, work_log=None):
        """Batched personalised PageRank; returns (V x k ranks, PrStats). work_log
        (2 x max_sweeps uint64) receives the cumulative (vertex updates, in-edge
        gathers) of the sources still iterating."""
        src = np.ascontiguousarray(sources, dtype=np.uint32) if isinstance(sources, (list, np.ndarray)) else sources
        k = int(src.shape[0])
        p = PrParams()
        _pr_default(C.byref(p))
        p.max_sweeps, p.teleport, p.damping, p.tol = max_sweeps, teleport, damping, tol
        p.flags = PR_TIME_SWEEPS if time_sweeps else 0
        if residuals is not None:
            p.residuals = ptr(residuals)
        if work_log is not None:
            p.work_log = ptr(work_log)
        if out is None:
            out = np.zeros((self.num_vertices, k), dtype=np.float32)
        st = PrStats()
        check(_ppr(self._h, ptr(src), k, C.byref(p), ptr(out), C.byref(st)))
        return out, st

    def warm_features(self, out=None):
        """(V, 8) float32 raw warm-start features (gcg_warm_features)."""
        if out is None:
            out = np.zeros((self.num_vertices, MLP_IN), dtype=np.float32)
        check(_warm_features(self._h, ptr(out)))
        return out

    def warm_start_rank(self, mlp, teleport=0.15, damping=0.85, out=None):
        """Learned initial ranks (gcg_warm_start_rank); returns (ranks, device ms)."""
        if out is None:
            out = np.zeros(self.num_vertices, dtype=np.float32)
        ms = C.c_double(0.0)
        check(_warm_start(self._h, mlp.handle, teleport, damping, ptr(out), C.byref(ms)))
        return out, ms.value

    def connected_components(self, out=None, algorithm=None, scheduler=False, max_iterations=0,
                             frontier_log=None):
        """Labels (minimum id per weak component) and CcStats; algorithm None = union-find."""
        if out is None:
            out = np.zeros(self.num_vertices, dtype=np.uint32)
        st = CcStats()
        if algorithm is None:
            check(_cc(self._h, ptr(out), C.byref(st)))
        else:
            p = CcParams(algorithm, 1 if scheduler else 0, max_iterations, 0, ptr(frontier_log))
            check(_cc_ex(self._h, C.byref(p), ptr(out), C.byref(st)))
        return out, st

    def triangle_count(self, per_rank=True, vertexmap=True):
        n = self.num_vertices
        pr = np.zeros(n, dtype=np.uint32) if per_rank is True else per_rank
        vm = np.zeros(n, dtype=np.uint32) if vertexmap is True else vertexmap
        tot = C.c_uint64(0)
        st = TcStats()
        check(_tc(self._h, C.byref(tot), ptr(pr) if pr is not None and pr is not False else None,
                  ptr(vm) if vm is not None and vm is not False else None, C.byref(st)))
        return int(tot.value), pr, vm, st


def parse_edgelist_file(path):
    m = _u64(0)
    check(_parse_file(os.fsencode(path), None, None, 0, C.byref(m)))
    src = np.zeros(max(1, m.value), dtype=np.uint32)
    dst = np.zeros(max(1, m.value), dtype=np.uint32)
    check(_parse_file(os.fsencode(path), ptr(src), ptr(dst), m.value, C.byref(m)))
    return src[: m.value], dst[: m.value]


def generate_rmat(scale, m, a=0.57, b=0.19, c=0.19, seed=1, src=None, dst=None):
    """R-MAT edges into src/dst (allocated as numpy if not given)."""
    if src is None:
        src = np.zeros(m, dtype=np.uint32)
        dst = np.zeros(m, dtype=np.uint32)
    check(_gen_rmat(scale, m, a, b, c, seed, ptr(src), ptr(dst)))
    return src, dst


def generate_er(n, m, seed=1, src=None, dst=None):
    if src is None:
        src = np.zeros(m, dtype=np.uint32)
        dst = np.zeros(m, dtype=np.uint32)
    check(_gen_er(n, m, seed, ptr(src), ptr(dst)))
    return src, dst


def write_vout(base, values):
    values = np.ascontiguousarray(values) if isinstance(values, np.ndarray) else values
    elem = values.dtype.itemsize if isinstance(values, np.ndarray) else values.element_size()
    n = values.shape[0]
    check(_write_vout(os.fsencode(base), ptr(values), n, elem))


def pagerank_csr_noalloc(in_rowptr, in_col, outdeg, out, num_vertices=None, max_sweeps=3, teleport=0.15,
                         damping=0.85, tol=0.0, init=1.0, stream=0, residuals=None):
    """gcg_pagerank_csr_noalloc: Jacobi PageRank over a CSR already in device
    memory (CUDA tensors), with no device allocation by the library.
    Returns PrStats; the ranks are written into ``out`` and, when given, each
    sweep's residual into the float64 device tensor ``residuals``."""
    n = int(out.shape[0]) if num_vertices is None else int(num_vertices)
    p = PrParams()
    _pr_default(C.byref(p))
    p.mode, p.max_sweeps, p.teleport, p.damping, p.tol, p.init = (PR_JACOBI, max_sweeps, teleport, damping, tol,
                                                                  init)
    if residuals is not None:
        p.residuals = ptr(residuals)
    st = PrStats()
    check(_pr_noalloc(ptr(in_rowptr), ptr(in_col), ptr(outdeg), n, C.byref(p), ptr(out), stream, C.byref(st)))
    return st


class Batch:
    """Many graphs solved by one persistent launch (gcg_batch_*)."""

    def __init__(self, graphs, one_hub=False):
        """one_hub: one shared-memory hub over the union's hottest sources, rows in
        id order (GCG_BATCH_ONE_HUB), instead of a hub per graph."""
        arr = (_vp * len(graphs))(*[g.handle for g in graphs])
        h = _vp()
        check(_batch_create(arr, len(graphs), BATCH_ONE_HUB if one_hub else 0, C.byref(h)))
        self._h = h
        self.ngraphs = len(graphs)
        off = np.zeros(len(graphs) + 1, dtype=np.uint64)
        check(_batch_offsets(h, ptr(off)))
        self.offsets = off

    def free(self):
        if self._h:
            _batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def set_stream(self, stream_ptr):
        check(_batch_set_stream(self._h, stream_ptr))

    def pagerank(self, max_sweeps=1000, teleport=0.15, damping=0.85, tol=0.0, init=1.0, init_rank=None, out=None,
                 flags=0):
        """Returns (ranks of all graphs concatenated, sweeps per graph, residual per graph, PrStats)."""
        p = PrParams()
        _pr_default(C.byref(p))
        p.max_sweeps, p.teleport, p.damping, p.tol, p.init, p.flags = (max_sweeps, teleport, damping, tol, init,
                                                                       flags)
        if init_rank is not None:
            init_rank = np.ascontiguousarray(init_rank, np.float32) if isinstance(init_rank, np.ndarray) else init_rank
            p.init_rank = ptr(init_rank)
        if out is None:
            out = np.zeros(int(self.offsets[-1]), dtype=np.float32)
        sweeps = np.zeros(self.ngraphs, dtype=np.int32)
        res = np.zeros(self.ngraphs, dtype=np.float64)
        st = PrStats()
        check(_batch_pagerank(self._h, C.byref(p), ptr(out), ptr(sweeps), ptr(res), C.byref(st)))
        return out, sweeps, res, st

    def autotune(self, sweeps=8):
        """Times the candidate launch configurations; returns (hub entries, queue run, ms per sweep)."""
        h, q, ms = _u32(0), _u32(0), C.c_double(0.0)
        check(_batch_autotune(self._h, sweeps, C.byref(h), C.byref(q), C.byref(ms)))
        return h.value, q.value, ms.value

    def set_config(self, hub_entries, queue_run):
        check(_batch_set_config(self._h, hub_entries, queue_run))

    def config(self):
        """(hub entries, queue run, captured solve ready)."""
        h, q, r = _u32(0), _u32(0), _i(0)
        check(_batch_get_config(self._h, C.byref(h), C.byref(q), C.byref(r)))
        return h.value, q.value, bool(r.value)

    def split(self, ranks):
        return [ranks[int(self.offsets[g]):int(self.offsets[g + 1])] for g in range(self.ngraphs)]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32) if isinstance(a, np.ndarray) else a


class Mlp:
    """The warm-start network (gcg_mlp_*): FP32 master weights on the device."""

    def __init__(self, seed=1):
        h = _vp()
        check(_mlp_create(seed, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def free(self):
        if self._h:
            _mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def get(self):
        """(params[MLP_NPARAMS], norm[16]) as float32 numpy arrays."""
        p = np.zeros(MLP_NPARAMS, np.float32)
        n = np.zeros(2 * MLP_IN, np.float32)
        check(_mlp_get(self._h, ptr(p), ptr(n)))
        return p, n

    def set(self, params=None, norm=None):
        params = None if params is None else np.ascontiguousarray(params, np.float32)
        norm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        check(_mlp_set(self._h, ptr(params), ptr(norm)))

    def fit_normalisation(self, x):
        x = _f32(x)
        check(_mlp_fit_norm(self._h, ptr(x), int(x.shape[0])))

    def forward(self, x, out=None):
        x = _f32(x)
        n = int(x.shape[0])
        if out is None:
            out = np.zeros(n, np.float32)
        check(_mlp_forward(self._h, ptr(x), n, ptr(out)))
        return out

    def gradient(self, x, t):
        """(gradient of mean squared error, mean loss) over all samples."""
        x, t = _f32(x), _f32(t)
        g = np.zeros(MLP_NPARAMS, np.float32)
        loss = C.c_double(0.0)
        check(_mlp_gradient(self._h, ptr(x), ptr(t), int(x.shape[0]), ptr(g), C.byref(loss)))
        return g, loss.value

    def train(self, x, t, epochs=None, batch=None, lr=None, seed=None):
        """Minibatch Adam; returns the mean training loss of each epoch."""
        x, t = _f32(x), _f32(t)
        p = MlpTrainParams()
        _mlp_train_default(C.byref(p))
        if epochs is not None:
            p.epochs = epochs
        if batch is not None:
            p.batch = batch
        if lr is not None:
            p.lr = lr
        if seed is not None:
            p.seed = seed
        losses = np.zeros(max(1, p.epochs), np.float32)
        check(_mlp_train(self._h, ptr(x), ptr(t), int(x.shape[0]), C.byref(p), ptr(losses)))
        return losses[: p.epochs]

    def save(self, path):
        p, n = self.get()
        np.savez(path, params=p, norm=n)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        m = cls(seed=0)
        m.set(z["params"], z["norm"])
        return m
