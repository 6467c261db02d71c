/*
 * Shared runtime pieces of libgcgpu: error state, pointer classification,
 * host<->device staging, the graph handle's destructor, synthetic generators,
 * and the vertex-value / metadata file writers.
 */
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gcg_internal.cuh"
#include "gcg_rng.h"

namespace gcg {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int status, const std::string &msg) {
    g_last_error = msg;
    return status;
}

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError(); /* clear: unregistered host pointer */
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int copy_in(void *dst_dev, const void *src_user, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return GCG_OK;
    GCG_CUDA(cudaMemcpyAsync(dst_dev, src_user, bytes, cudaMemcpyDefault, s));
    return GCG_OK;
}

int copy_out(void *dst_user, const void *src_dev, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return GCG_OK;
    GCG_CUDA(cudaMemcpyAsync(dst_user, src_dev, bytes, cudaMemcpyDefault, s));
    if (!is_device_ptr(dst_user)) GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

void pool_keep_memory() {
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return;
    }
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    done[dev] = true;
}

int num_sms() {
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
        cached = n;
    }
    return cached;
}

/* ---- generators --------------------------------------------------------- */

static gcg_rmat_thresholds rmat_thresholds(double a, double b, double c) {
    const double two32 = 4294967296.0;
    gcg_rmat_thresholds t;
    t.ta = (uint64_t)(a * two32);
    t.tab = (uint64_t)((a + b) * two32);
    t.tabc = (uint64_t)((a + b + c) * two32);
    return t;
}

__global__ void k_rmat(uint64_t key, uint64_t m, uint32_t scale, gcg_rmat_thresholds t, uint32_t *src,
                       uint32_t *dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        gcg_rmat_edge(key, i, scale, t, &s, &d);
        src[i] = s;
        dst[i] = d;
    }
}

__global__ void k_er(uint64_t key, uint64_t m, uint32_t n, uint32_t *src, uint32_t *dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        gcg_er_edge(key, i, n, &s, &d);
        src[i] = s;
        dst[i] = d;
    }
}

template <typename F>
static void host_parallel_for(uint64_t m, F f) {
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (m < 65536) nt = 1;
    std::vector<std::thread> th;
    uint64_t chunk = (m + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        uint64_t b = t * chunk, e = std::min(m, b + chunk);
        if (b >= e) break;
        th.emplace_back([=]() {
            for (uint64_t i = b; i < e; ++i) f(i);
        });
    }
    for (auto &x : th) x.join();
}

}  // namespace gcg

gcg_graph::~gcg_graph() {
    delete plan;
    gcg::free_chunk_plan(cplan);
    gcg::free_ppr_plan(pplan);
    free(intervals_host);
}

using namespace gcg;

extern "C" {

const char *gcg_last_error(void) { return g_last_error.c_str(); }

const char *gcg_version(void) { return "gcgpu 0.1 (sm_100a)"; }

int gcg_generate_rmat(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed,
                      uint32_t *src, uint32_t *dst) {
    if (!src || !dst) return fail(GCG_ERR_INVALID, "gcg_generate_rmat: null output");
    if (scale == 0 || scale > 32) return fail(GCG_ERR_INVALID, "gcg_generate_rmat: scale must be 1..32");
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return fail(GCG_ERR_INVALID, "gcg_generate_rmat: bad a/b/c");
    gcg_rmat_thresholds t = rmat_thresholds(a, b, c);
    uint64_t key = gcg_seed_key(seed);
    bool dev = is_device_ptr(src), dev2 = is_device_ptr(dst);
    if (dev != dev2) return fail(GCG_ERR_INVALID, "gcg_generate_rmat: src and dst must both be host or device");
    if (dev) {
        if (m == 0) return GCG_OK;
        unsigned blocks = (unsigned)std::min<uint64_t>((m + 255) / 256, (uint64_t)num_sms() * 16);
        k_rmat<<<blocks, 256>>>(key, m, scale, t, src, dst);
        GCG_LAUNCH_CHECK();
        GCG_CUDA(cudaDeviceSynchronize());
        return GCG_OK;
    }
    host_parallel_for(m, [&](uint64_t i) { gcg_rmat_edge(key, i, scale, t, src + i, dst + i); });
    return GCG_OK;
}

int gcg_generate_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *src, uint32_t *dst) {
    if (!src || !dst) return fail(GCG_ERR_INVALID, "gcg_generate_er: null output");
    if (n == 0) return fail(GCG_ERR_INVALID, "gcg_generate_er: n must be > 0");
    uint64_t key = gcg_seed_key(seed);
    bool dev = is_device_ptr(src), dev2 = is_device_ptr(dst);
    if (dev != dev2) return fail(GCG_ERR_INVALID, "gcg_generate_er: src and dst must both be host or device");
    if (dev) {
        if (m == 0) return GCG_OK;
        unsigned blocks = (unsigned)std::min<uint64_t>((m + 255) / 256, (uint64_t)num_sms() * 16);
        k_er<<<blocks, 256>>>(key, m, n, src, dst);
        GCG_LAUNCH_CHECK();
        GCG_CUDA(cudaDeviceSynchronize());
        return GCG_OK;
    }
    host_parallel_for(m, [&](uint64_t i) { gcg_er_edge(key, i, n, src + i, dst + i); });
    return GCG_OK;
}

int gcg_write_vout(const char *base, const void *values, uint32_t num_vertices, uint32_t elem_size) {
    if (!base || !values || elem_size == 0) return fail(GCG_ERR_INVALID, "gcg_write_vout: bad argument");
    size_t bytes = (size_t)num_vertices * elem_size;
    std::vector<char> host;
    const void *src = values;
    if (is_device_ptr(values)) {
        host.resize(bytes);
        GCG_CUDA(cudaMemcpy(host.data(), values, bytes, cudaMemcpyDeviceToHost));
        src = host.data();
    }
    /* <base>.<sizeof(VT)>B.vout (src/api/chifilenames.hpp:65-71): a raw array */
    std::string fname = std::string(base) + "." + std::to_string(elem_size) + "B.vout";
    FILE *f = fopen(fname.c_str(), "wb");
    if (!f) return fail(GCG_ERR_IO, "cannot write " + fname);
    size_t w = fwrite(src, 1, bytes, f);
    fclose(f);
    if (w != bytes) return fail(GCG_ERR_IO, "short write to " + fname);
    return GCG_OK;
}

int gcg_graph_set_stream(gcg_graph *g, void *stream) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_graph_set_stream: null graph");
    g->stream = (cudaStream_t)stream;
    return GCG_OK;
}

int gcg_graph_free(gcg_graph *g) {
    if (!g) return GCG_OK;
    cudaStreamSynchronize(g->stream);
    delete g;
    return GCG_OK;
}

int gcg_graph_get_device_view(const gcg_graph *g, gcg_graph_device_view *v) {
    if (!g || !v) return fail(GCG_ERR_INVALID, "gcg_graph_get_device_view: null argument");
    v->in_rowptr = g->in_rowptr.get();
    v->in_col = g->in_col.get();
    v->out_rowptr = g->has_out ? g->out_rowptr.get() : nullptr;
    v->out_col = g->has_out ? g->out_col.get() : nullptr;
    v->indeg = g->indeg.get();
    v->outdeg = g->outdeg.get();
    v->num_vertices = g->nv;
    v->reserved = 0;
    v->num_edges = g->ne;
    v->stream = (void *)g->stream;
    return GCG_OK;
}

int gcg_graph_get_info(const gcg_graph *g, gcg_graph_info *info) {
    if (!g || !info) return fail(GCG_ERR_INVALID, "gcg_graph_get_info: null argument");
    info->num_vertices = g->nv;
    info->nshards = g->nshards;
    info->num_edges = g->ne;
    info->has_out_csr = g->has_out ? 1u : 0u;
    info->reserved = 0;
    return GCG_OK;
}

}  // extern "C"
