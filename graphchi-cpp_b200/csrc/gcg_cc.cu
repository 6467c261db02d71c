/*
 * Connected components: replaces graphchi_engine::run(ConnectedComponentsProgram)
 * (example_apps/connectedcomponents.cpp:79-138), whose fixpoint labels every
 * vertex with the minimum vertex id of its weakly connected component.
 *
 * Device form: min-label propagation on roots with pointer-jumping shortcuts
 * (hook-and-compress). parent[v] starts at v; every edge (u,v) hooks the larger
 * of the two current roots under the smaller with a CAS (labels only move to
 * smaller ids, so parent[x] <= x always holds and each final root is the
 * minimum id of its component); finds shorten paths by pointer jumping (path
 * halving) as they go; a last pass jumps every vertex to its root. The edge pass
 * walks the merge-path tiles of the in-CSR, so hubs and empty rows are spread
 * evenly over the CTAs; one pass suffices because hooking is transitive.
 * The CAS loop has no waits on other threads: each failed CAS moves to a
 * strictly smaller id, so it ends.
 *
 * When every vertex's full neighbourhood is at hand (a symmetrised graph: the
 * in-list; otherwise the in-list plus the out-list), the edge pass samples
 * instead (the Afforest scheme): one pass links each vertex to its first
 * neighbour, then the roots of 1024 sampled vertices name the most frequent
 * one (the giant component); only vertices whose root is not it link their
 * remaining neighbours (a thread per short list, a warp per long one). A skipped vertex of
 * the giant component loses nothing: each of its other edges is also in the
 * neighbour's list, and that neighbour links it unless it is in the giant
 * component too. The same hook keeps the labels (the minimum id per component).
 */
#include <algorithm>

#include "gcg_internal.cuh"
#include "gcg_mergepath.cuh"

namespace gcg {
namespace {

__device__ __forceinline__ uint32_t find_root(uint32_t *parent, uint32_t x) {
    uint32_t p = ((volatile uint32_t *)parent)[x];
    while (p != x) {
        uint32_t gp = ((volatile uint32_t *)parent)[p];
        if (gp != p) ((volatile uint32_t *)parent)[x] = gp; /* path halving: gp < p <= x */
        x = p;
        p = gp;
    }
    return x;
}

__device__ __forceinline__ void hook(uint32_t *parent, uint32_t u, uint32_t v) {
    uint32_t a = find_root(parent, u);
    uint32_t b = find_root(parent, v);
    while (a != b) {
        uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
        uint32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) return;
        /* hi was hooked elsewhere meanwhile: continue from its new parent */
        a = find_root(parent, old);
        b = lo == a ? a : find_root(parent, lo);
    }
}

__global__ void k_cc_init(uint32_t nv, uint32_t *parent) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) parent[v] = v;
}

__global__ void __launch_bounds__(MP_THREADS) k_cc_hook(const uint32_t *__restrict__ rowptr,
                                                        const uint32_t *__restrict__ col,
                                                        const uint32_t *__restrict__ tile_row,
                                                        const uint32_t *__restrict__ tile_edge, uint32_t ntiles,
                                                        uint32_t *parent) {
    __shared__ uint32_t s_rowend[MP_TILE];
    __shared__ uint32_t s_src[MP_TILE];
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t r0 = tile_row[t], r1 = tile_row[t + 1];
        const uint32_t e0 = tile_edge[t], e1 = tile_edge[t + 1];
        const uint32_t nrows = r1 - r0, nedges = e1 - e0;
        for (uint32_t k = threadIdx.x; k < nrows; k += MP_THREADS) s_rowend[k] = rowptr[r0 + k + 1] - e0;
        for (uint32_t k = threadIdx.x; k < nedges; k += MP_THREADS) s_src[k] = __ldg(col + e0 + k);
        __syncthreads();
        const uint32_t items = nrows + nedges;
        const uint32_t d0 = min((uint32_t)threadIdx.x * MP_ITEMS, items);
        const uint32_t d1 = min(d0 + MP_ITEMS, items);
        uint32_t ti = mp_search(s_rowend, nrows, nedges, d0);
        uint32_t tj = d0 - ti;
        for (uint32_t d = d0; d < d1; ++d) {
            if (ti < nrows && s_rowend[ti] <= tj) {
                ++ti;
            } else {
                hook(parent, s_src[tj], r0 + ti);
                ++tj;
            }
        }
        __syncthreads();
    }
}

/* neighbour i of v in the concatenation in-list(v) ++ out-list(v) (rout NULL: in-list only) */
struct Nbrs {
    const uint32_t *rin, *cin, *rout, *cout;
};
__device__ __forceinline__ uint32_t nbr_count(const Nbrs &n, uint32_t v) {
    uint32_t d = n.rin[v + 1] - n.rin[v];
    if (n.rout) d += n.rout[v + 1] - n.rout[v];
    return d;
}
__device__ __forceinline__ uint32_t nbr_at(const Nbrs &n, uint32_t v, uint32_t i) {
    const uint32_t b = n.rin[v], din = n.rin[v + 1] - b;
    return i < din ? n.cin[b + i] : n.cout[n.rout[v] + (i - din)];
}

/* Link of the sampling scheme: climbs one parent at a time and re-reads the
 * larger side's parent before the CAS, so a pair already joined by another
 * thread ends without an atomic (hub roots see many such pairs). Like hook, it
 * only ever points a root at a smaller id. */
__device__ __forceinline__ void link(uint32_t *parent, uint32_t u, uint32_t v) {
    volatile uint32_t *p = parent;
    uint32_t p1 = p[u], p2 = p[v];
    while (p1 != p2) {
        const uint32_t hi = p1 > p2 ? p1 : p2, lo = p1 > p2 ? p2 : p1;
        const uint32_t ph = p[hi];
        if (ph == lo) return;
        if (ph == hi && atomicCAS(parent + hi, hi, lo) == hi) return;
        p1 = p[p[hi]];
        p2 = p[lo];
    }
}

/* sampling round: link v to its first CC_ROUNDS neighbours (adjacent in the
 * list, so one sector of the column array per vertex) */
constexpr uint32_t CC_ROUNDS = 1;
__device__ __forceinline__ uint32_t find_root_ro(const uint32_t *parent, uint32_t x);
__global__ void k_cc_rounds(Nbrs n, uint32_t nv, uint32_t *parent) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t d = nbr_count(n, v);
#pragma unroll
        for (uint32_t r = 0; r < CC_ROUNDS; ++r)
            if (r < d) link(parent, v, nbr_at(n, v, r));
    }
}

/* the most frequent root among 1024 sampled vertices (ties: the smaller id);
 * one block of 1024 threads: bitonic sort in shared memory, then each run's
 * length from two binary searches by its first thread */
__global__ void __launch_bounds__(1024) k_cc_sample(const uint32_t *parent, uint32_t nv, uint32_t *giant) {
    __shared__ uint32_t s[1024];
    __shared__ unsigned long long s_best;
    const uint32_t t = threadIdx.x;
    uint64_t z = (uint64_t)t * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    s[t] = find_root_ro(parent, (uint32_t)(z % nv));
    if (t == 0) s_best = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= 1024; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = t ^ j;
            if (o > t) {
                const uint32_t x = s[t], y = s[o];
                const bool up = (t & k) == 0;
                if ((x > y) == up) {
                    s[t] = y;
                    s[o] = x;
                }
            }
            __syncthreads();
        }
    /* run starting at t: key = (1024 - length) << 32 | value, smallest wins; the
     * run ends at the first entry above s[t] */
    if (t == 0 || s[t] != s[t - 1]) {
        const uint32_t x = s[t];
        uint32_t lo = t + 1, hi = 1024;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s[mid] > x) hi = mid; else lo = mid + 1;
        }
        atomicMin(&s_best, ((unsigned long long)(1024u - (lo - t)) << 32) | x);
    }
    __syncthreads();
    if (t == 0) *giant = (uint32_t)(s_best & 0xFFFFFFFFull);
}

constexpr uint32_t CC_THREAD_MAX = 64; /* remaining neighbours a thread links itself */

/* vertices outside the giant component link their remaining neighbours */
__global__ void k_cc_rest(Nbrs n, uint32_t nv, const uint32_t *giant, uint32_t *parent, uint32_t *work,
                          uint32_t *nwork) {
    const uint32_t c = *giant;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t d = nbr_count(n, v);
        if (d <= CC_ROUNDS || find_root(parent, v) == c) continue;
        if (d - CC_ROUNDS <= CC_THREAD_MAX) {
            for (uint32_t i = CC_ROUNDS; i < d; ++i) link(parent, v, nbr_at(n, v, i));
        } else {
            work[atomicAdd(nwork, 1u)] = v;
        }
    }
}

__global__ void k_cc_rest_long(Nbrs n, const uint32_t *work, const uint32_t *nwork, uint32_t *parent) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = *nwork;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nw; k += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t v = work[k], d = nbr_count(n, v);
        for (uint32_t i = CC_ROUNDS + lane; i < d; i += 32u) link(parent, v, nbr_at(n, v, i));
    }
}

/* Final pass: every vertex jumps to its root. The find here only reads (no path
 * halving): a halving store racing with another vertex's final store could put
 * a non-root ancestor back. The only stores are parent[v] = root(v) by v's own
 * thread, and a root is an ancestor, so concurrent readers stay correct. */
__device__ __forceinline__ uint32_t find_root_ro(const uint32_t *parent, uint32_t x) {
    uint32_t p = ((const volatile uint32_t *)parent)[x];
    while (p != x) {
        x = p;
        p = ((const volatile uint32_t *)parent)[x];
    }
    return x;
}

__global__ void k_cc_compress(uint32_t nv, uint32_t *parent, uint32_t *nroots) {
    uint32_t roots = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t r = find_root_ro(parent, v);
        ((volatile uint32_t *)parent)[v] = r;
        roots += (r == v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) roots += __shfl_down_sync(0xFFFFFFFFu, roots, o);
    if ((threadIdx.x & 31) == 0 && roots) atomicAdd(nroots, roots);
}

}  // namespace
}  // namespace gcg

using namespace gcg;

extern "C" int gcg_connected_components(gcg_graph *g, uint32_t *labels, gcg_cc_stats *stats) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_connected_components: null graph");
    GCG_TRY(ensure_plan(g));
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    const PrPlan &pl = *g->plan;
    tbuf<uint32_t> parent_tmp, cnt;
    uint32_t *parent;
    const bool dev_out = labels && is_device_ptr(labels);
    if (dev_out) {
        parent = labels;
    } else {
        GCG_TRY(parent_tmp.alloc(nv, s));
        parent = parent_tmp.get();
    }
    /* sampling needs each vertex's whole neighbourhood: symmetric in-lists, or in + out lists */
    const bool sampled = nv > 0 && (g->symmetric || g->has_out);
    tbuf<uint32_t> work;
    GCG_TRY(cnt.alloc(4, s));
    GCG_CUDA(cudaMemsetAsync(cnt.get(), 0, 16, s));
    if (sampled) GCG_TRY(work.alloc(std::max<uint32_t>(nv, 1), s));
    unsigned vb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, (uint64_t)num_sms() * 16));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cc_hook, MP_THREADS, 0) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        per_sm = 4;
    }
    unsigned tb = (unsigned)std::max<uint32_t>(1, std::min<uint32_t>(pl.ntiles, (uint32_t)(num_sms() * per_sm)));
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    k_cc_init<<<vb, 256, 0, s>>>(nv, parent);
    if (sampled) {
        Nbrs nb;
        nb.rin = g->in_rowptr.get();
        nb.cin = g->in_col.get();
        nb.rout = g->symmetric ? nullptr : g->out_rowptr.get();
        nb.cout = g->symmetric ? nullptr : g->out_col.get();
        k_cc_rounds<<<vb, 256, 0, s>>>(nb, nv, parent);
        k_cc_sample<<<1, 1024, 0, s>>>(parent, nv, cnt.get() + 1);
        k_cc_rest<<<vb, 256, 0, s>>>(nb, nv, cnt.get() + 1, parent, work.get(), cnt.get() + 2);
        k_cc_rest_long<<<num_sms() * 8, 256, 0, s>>>(nb, work.get(), cnt.get() + 2, parent);
    } else {
        k_cc_hook<<<tb, MP_THREADS, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), pl.tile_row.get(),
                                           pl.tile_edge.get(), pl.ntiles, parent);
    }
    k_cc_compress<<<vb, 256, 0, s>>>(nv, parent, cnt.get());
    GCG_LAUNCH_CHECK();
    GCG_CUDA(cudaEventRecord(ev1, s));
    uint32_t nroots = 0;
    GCG_CUDA(cudaMemcpyAsync(&nroots, cnt.get(), 4, cudaMemcpyDeviceToHost, s));
    if (labels && !dev_out) GCG_TRY(copy_out(labels, parent, (size_t)nv * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (stats) {
        stats->passes = sampled ? 2 : 1;
        stats->ncomponents = nroots;
        stats->device_ms = ms;
    }
    return GCG_OK;
}

extern "C" int gcg_connected_components_ex(gcg_graph *g, const gcg_cc_params *p, uint32_t *labels,
                                           gcg_cc_stats *stats) {
    if (!g || !p) return fail(GCG_ERR_INVALID, "gcg_connected_components_ex: null argument");
    if (p->algorithm == GCG_CC_UNION_FIND) return gcg_connected_components(g, labels, stats);
    if (p->algorithm != GCG_CC_LABEL_PROPAGATION)
        return fail(GCG_ERR_INVALID, "gcg_connected_components_ex: unknown algorithm");
    const int iters = p->max_iterations > 0 ? p->max_iterations : 1000;
    return cc_label_propagation(g, p->scheduler, iters, labels, stats, p->frontier_log);
}
