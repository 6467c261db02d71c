/*
 * Shared runtime pieces of libgcgpu: error state, pointer classification,
 * host<->device staging, the graph handle's destructor, synthetic generators,
 * and the vertex-value / metadata file writers.
 */
#include <stdio.h>
#include <string.h>

#include <stdlib.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>
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

static bool g_pool_kept[64] = {false}; /* devices whose default pool keeps freed memory */

void pool_keep_memory() {
    bool *done = g_pool_kept;
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

/* ---- block cache ----------------------------------------------------------
 * Graph builds, chunk plans and solver workspaces ask for the same sizes again
 * and again (a loop that builds, solves and frees a graph per input), and
 * cudaMalloc/cudaFree cost 0.3-5 ms apiece at these sizes. A freed block waits
 * in an idle list keyed by (device, size class) for the next request of its
 * class. Before a block enters the list its device is synchronised, which is
 * what cudaFree did, so no kernel still touches a block that is handed out
 * again. Classes: 512-byte multiples up to 1 MiB, 2 MiB multiples above. */
namespace {

constexpr int CACHE_DEVS = 64;
constexpr int HOST_DEV = -1;

struct BlockCache {
    std::mutex mu;
    std::unordered_map<void *, std::pair<size_t, int>> live; /* ptr -> (class bytes, device or HOST_DEV) */
    std::multimap<std::pair<int, size_t>, void *> idle;
    size_t idle_dev[CACHE_DEVS] = {0};
    size_t cap_dev[CACHE_DEVS] = {0};
    bool cap_known[CACHE_DEVS] = {false};
    size_t idle_host = 0, cap_host = 0;
    bool host_cap_known = false;
};

/* never destroyed: blocks may be returned by static destructors after main */
BlockCache &cache() {
    static BlockCache *c = new BlockCache();
    return *c;
}

size_t size_class(size_t b) {
    if (b == 0) b = 1;
    if (b <= ((size_t)1 << 20)) return (b + 511) & ~(size_t)511;
    const size_t g = (size_t)2 << 20;
    return (b + g - 1) & ~(g - 1);
}

size_t env_mb(const char *name, size_t dflt) {
    const char *v = getenv(name);
    if (!v || !*v) return dflt;
    char *end = nullptr;
    unsigned long long mb = strtoull(v, &end, 10);
    if (end == v) return dflt;
    return (size_t)mb << 20;
}

/* under the lock */
size_t device_cap(BlockCache &c, int dev) {
    if (!c.cap_known[dev]) {
        size_t freeb = 0, total = 0;
        if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
            cudaGetLastError();
            total = 0;
        }
        c.cap_dev[dev] = env_mb("GCG_DEVICE_CACHE_MB", total / 4);
        c.cap_known[dev] = true;
    }
    return c.cap_dev[dev];
}

size_t host_cap(BlockCache &c) {
    if (!c.host_cap_known) {
        c.cap_host = env_mb("GCG_HOST_CACHE_MB", (size_t)256 << 20);
        c.host_cap_known = true;
    }
    return c.cap_host;
}

/* frees idle blocks: of device dev_sel (>= 0), of every device (ALL_DEVS) or of
 * none (NO_DEVS), and the host's with host; returns the bytes released */
constexpr int ALL_DEVS = -1, NO_DEVS = -2;
uint64_t drain(int dev_sel, bool host) {
    BlockCache &c = cache();
    std::vector<std::pair<int, void *>> victims;
    uint64_t bytes = 0;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.idle.begin(); it != c.idle.end();) {
            const int d = it->first.first;
            const bool take = d == HOST_DEV ? host : (dev_sel == ALL_DEVS || d == dev_sel);
            if (!take) {
                ++it;
                continue;
            }
            bytes += it->first.second;
            if (d == HOST_DEV)
                c.idle_host -= it->first.second;
            else
                c.idle_dev[d] -= it->first.second;
            victims.emplace_back(d, it->second);
            it = c.idle.erase(it);
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto &v : victims) {
        if (v.first == HOST_DEV) {
            cudaFreeHost(v.second);
        } else {
            if (v.first != cur) cudaSetDevice(v.first);
            cudaFree(v.second);
            if (v.first != cur) cudaSetDevice(cur);
        }
    }
    cudaGetLastError();
    return bytes;
}

}  // namespace

/* Out of device memory: the idle blocks of the current device go back to the
 * driver and its default pool drops the memory it keeps for freed temporaries. */
void reclaim_device_memory() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    drain(dev, false);
    cudaMemPool_t pool;
    if (cudaDeviceSynchronize() == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
}

namespace {

cudaError_t cached_alloc(void **p, size_t bytes, bool host) {
    *p = nullptr;
    int dev = HOST_DEV;
    if (!host) {
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= CACHE_DEVS) return cudaMalloc(p, bytes);
    }
    const size_t cls = size_class(bytes);
    BlockCache &c = cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (!host) device_cap(c, dev); /* read while dev is the current device */
        auto it = c.idle.find({dev, cls});
        if (it != c.idle.end()) {
            *p = it->second;
            c.idle.erase(it);
            if (host)
                c.idle_host -= cls;
            else
                c.idle_dev[dev] -= cls;
            c.live[*p] = {cls, dev};
            return cudaSuccess;
        }
    }
    cudaError_t e = host ? cudaMallocHost(p, cls) : cudaMalloc(p, cls);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        if (host)
            drain(NO_DEVS, true);
        else
            reclaim_device_memory();
        e = host ? cudaMallocHost(p, cls) : cudaMalloc(p, cls);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[*p] = {cls, dev};
    return cudaSuccess;
}

void cached_free(void *p, bool host) {
    if (!p) return;
    BlockCache &c = cache();
    size_t cls = 0;
    int dev = HOST_DEV;
    bool keep = false;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.live.find(p);
        if (it != c.live.end()) {
            cls = it->second.first;
            dev = it->second.second;
            c.live.erase(it);
            const size_t cap = dev == HOST_DEV ? host_cap(c) : device_cap(c, dev);
            const size_t held = dev == HOST_DEV ? c.idle_host : c.idle_dev[dev];
            keep = held + cls <= cap;
        } else {
            dev = host ? HOST_DEV : -2; /* not ours: hand straight back */
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    const int sync_dev = dev >= 0 ? dev : cur;
    if (sync_dev != cur) cudaSetDevice(sync_dev);
    if (keep) {
        /* what cudaFree/cudaFreeHost would wait for: no kernel or copy still uses p */
        keep = cudaDeviceSynchronize() == cudaSuccess;
        if (keep) {
            std::lock_guard<std::mutex> lk(c.mu);
            c.idle.insert({{dev, cls}, p});
            if (dev == HOST_DEV)
                c.idle_host += cls;
            else
                c.idle_dev[dev] += cls;
        }
    }
    if (!keep) {
        if (host)
            cudaFreeHost(p);
        else
            cudaFree(p);
    }
    if (sync_dev != cur) cudaSetDevice(cur);
    cudaGetLastError();
}

}  // namespace

cudaError_t dev_alloc(void **p, size_t bytes) { return cached_alloc(p, bytes, false); }
void dev_free(void *p) { cached_free(p, false); }
cudaError_t host_alloc(void **p, size_t bytes) { return cached_alloc(p, bytes, true); }
void host_free(void *p) { cached_free(p, true); }

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
    gcg::free_gs_plan(gsplan);
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

int gcg_cached_memory(uint64_t *idle_device_bytes, uint64_t *idle_host_bytes) {
    BlockCache &c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    uint64_t d = 0;
    for (int i = 0; i < CACHE_DEVS; ++i) d += c.idle_dev[i];
    if (idle_device_bytes) *idle_device_bytes = d;
    if (idle_host_bytes) *idle_host_bytes = c.idle_host;
    return GCG_OK;
}

int gcg_release_cached_memory(uint64_t *released_bytes) {
    const uint64_t b = drain(ALL_DEVS, true);
    if (released_bytes) *released_bytes = b;
    /* and the stream-ordered temporaries kept by the default pools */
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess) {
        for (int d = 0; d < 64; ++d) {
            if (!g_pool_kept[d]) continue;
            cudaMemPool_t pool;
            if (cudaSetDevice(d) == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
                cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess)
                cudaMemPoolTrimTo(pool, 0);
        }
        cudaSetDevice(cur);
    }
    cudaGetLastError();
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
