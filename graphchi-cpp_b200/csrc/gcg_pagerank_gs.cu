/*
 * Exact vertex-API PageRank: the in-memory program of example_apps/pagerank.cpp
 * (:121-146) as the engine runs it with deterministic parallelism
 * (src/engine/graphchi_engine.hpp:396-454): one Gauss-Seidel sweep per iteration
 * in ascending vertex id order, each vertex reading the values its smaller-id
 * in-neighbours wrote in this sweep and its larger-id in-neighbours' values from
 * the previous sweep, summing them in ascending source order in float.
 *
 * Parallel form: vertex v depends on in-neighbours u < v only, so v's level
 * (1 + max level of those u, 0 if none) orders the sweep: every level is a set of
 * independent vertices. Within a sweep, levels run in order; each vertex sums
 * sequentially (bit-exact float order), reading new values below its id and old
 * values above it. Levels come from a monotone relaxation over the in-CSR and a
 * radix sort of (level, id); the per-level launches of one sweep are captured
 * once in a CUDA graph and replayed per sweep.
 */
#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

__global__ void k_level_relax(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                              uint32_t *level, int *changed) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t l = 0;
        for (uint32_t j = rowptr[v]; j < rowptr[v + 1]; ++j) {
            uint32_t u = col[j];
            if (u >= v) break; /* sources ascending */
            uint32_t lu = ((volatile uint32_t *)level)[u] + 1u;
            l = lu > l ? lu : l;
        }
        if (l > level[v]) {
            level[v] = l;
            *changed = 1;
        }
    }
}

__global__ void k_level_keys(const uint32_t *__restrict__ level, uint32_t nv, uint32_t vbits, uint64_t *keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)level[v] << vbits) | v;
}

__global__ void k_level_bounds(const uint64_t *__restrict__ keys, uint32_t nv, uint32_t vbits, uint32_t nlev,
                               uint32_t *__restrict__ off, uint32_t *__restrict__ order) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        order[i] = (uint32_t)(k & mask);
        int64_t l = (int64_t)(k >> vbits);
        int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> vbits);
        for (int64_t x = prev + 1; x <= l; ++x) off[x] = i;
        if (i == nv - 1)
            for (int64_t x = l + 1; x <= (int64_t)nlev; ++x) off[x] = nv;
    }
}

__global__ void k_max_u32(const uint32_t *__restrict__ a, uint32_t n, uint32_t *out) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

/* pagerank.cpp:124,137-139: pr starts at 0.15; iteration 0 sets 1/outc when outc > 0 */
__global__ void k_gs_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float reset, float *pr) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t oc = outdeg[v];
        pr[v] = oc > 0 ? __fdiv_rn(1.0f, (float)oc) : reset;
    }
}

/* pagerank.cpp:127-136 for the vertices of one level */
__global__ void k_gs_level(const uint32_t *__restrict__ order, uint32_t begin, uint32_t end,
                           const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col,
                           const uint32_t *__restrict__ outdeg, const float *__restrict__ pr_old, float *pr_new,
                           double reset, double damping) {
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const uint32_t v = order[i];
        float sum = 0.0f;
        const uint32_t jb = rowptr[v], je = rowptr[v + 1];
        for (uint32_t j = jb; j < je; ++j) {
            const uint32_t u = __ldg(col + j);
            sum += (u < v) ? ((volatile const float *)pr_new)[u] : __ldg(pr_old + u);
        }
        /* explicit round-to-nearest ops: no FMA contraction, the same rounding as
         * the reference's separate double multiply and add */
        const int outc = (int)outdeg[v];
        const double t = __dadd_rn(reset, __dmul_rn(damping, (double)sum));
        pr_new[v] = outc > 0 ? (float)__ddiv_rn(t, (double)outc) : (float)t;
    }
}

/* pagerank.cpp:140-143: the stored value is pr * outc on the last iteration */
__global__ void k_gs_final(uint32_t nv, const uint32_t *__restrict__ outdeg, const float *__restrict__ pr, float *out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t oc = outdeg[v];
        out[v] = oc > 0 ? __fmul_rn(pr[v], (float)oc) : pr[v];
    }
}

inline unsigned vgrid(uint32_t n) {
    uint64_t b = ((uint64_t)n + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * 16;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

/* Level schedule of the id-ordered dependency DAG: order[] (vertices by
 * (level, id)) and off[l] = first index of level l, nlev levels. */
struct GsPlan {
    uint32_t nlev = 0;
    dbuf<uint32_t> order;
    std::vector<uint32_t> off;
};

static int build_gs_plan(gcg_graph *g, GsPlan &pl) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    tbuf<uint32_t> level;
    tbuf<int> changed;
    GCG_TRY(level.alloc(nv, s));
    GCG_TRY(changed.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(level.get(), 0, (size_t)nv * 4, s));
    for (int it = 0;; ++it) {
        int h = 0;
        GCG_CUDA(cudaMemsetAsync(changed.get(), 0, sizeof(int), s));
        k_level_relax<<<vgrid(nv), 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), nv, level.get(), changed.get());
        GCG_LAUNCH_CHECK();
        GCG_CUDA(cudaMemcpyAsync(&h, changed.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        if (!h) break;
        if (it > (int)nv + 1) return fail(GCG_ERR_CUDA, "level relaxation did not converge");
    }
    tbuf<uint32_t> dmax;
    GCG_TRY(dmax.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(dmax.get(), 0, 4, s));
    k_max_u32<<<vgrid(nv), 256, 0, s>>>(level.get(), nv, dmax.get());
    uint32_t maxl = 0;
    GCG_CUDA(cudaMemcpyAsync(&maxl, dmax.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    pl.nlev = maxl + 1;
    uint32_t lbits = 1;
    while (lbits < 32 && (1ull << lbits) <= maxl) ++lbits;
    tbuf<uint64_t> keys, tmp;
    GCG_TRY(keys.alloc(nv, s));
    GCG_TRY(tmp.alloc(nv, s));
    k_level_keys<<<vgrid(nv), 256, 0, s>>>(level.get(), nv, g->vbits, keys.get());
    uint64_t *sorted = nullptr;
    GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nv, (int)g->vbits, (int)(g->vbits + lbits), &sorted, s));
    tbuf<uint32_t> doff;
    GCG_TRY(doff.alloc((size_t)pl.nlev + 1, s));
    GCG_TRY(pl.order.alloc(nv));
    k_level_bounds<<<vgrid(nv), 256, 0, s>>>(sorted, nv, g->vbits, pl.nlev, doff.get(), pl.order.get());
    GCG_LAUNCH_CHECK();
    pl.off.resize((size_t)pl.nlev + 1);
    GCG_CUDA(cudaMemcpyAsync(pl.off.data(), doff.get(), ((size_t)pl.nlev + 1) * 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

int pagerank_gs_exact(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    GsPlan pl;
    GCG_TRY(build_gs_plan(g, pl));
    tbuf<float> pr;
    GCG_TRY(pr.alloc((size_t)2 * nv, s));
    float *pr_old = pr.get(), *pr_new = pr.get() + nv;
    const float reset = (float)p->teleport;
    k_gs_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), reset, pr_old);
    GCG_LAUNCH_CHECK();

    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    /* one sweep = all levels in order, then pr_old <- pr_new; captured once */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap;
    GCG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    GCG_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    for (uint32_t l = 0; l < pl.nlev; ++l) {
        uint32_t b = pl.off[l], e = pl.off[l + 1];
        if (b == e) continue;
        k_gs_level<<<vgrid(e - b), 256, 0, cap>>>(pl.order.get(), b, e, g->in_rowptr.get(), g->in_col.get(),
                                                 g->outdeg.get(), pr_old, pr_new, p->teleport, p->damping);
    }
    cudaMemcpyAsync(pr_old, pr_new, (size_t)nv * 4, cudaMemcpyDeviceToDevice, cap);
    cudaError_t ce = cudaStreamEndCapture(cap, &graph);
    if (ce != cudaSuccess) {
        cudaStreamDestroy(cap);
        return fail(GCG_ERR_CUDA, std::string("sweep capture: ") + cudaGetErrorString(ce));
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaStreamDestroy(cap);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(GCG_ERR_CUDA, std::string("sweep graph instantiate: ") + cudaGetErrorString(ce));
    }
    GCG_CUDA(cudaEventRecord(ev0, s));
    for (int sw = 0; sw < p->max_sweeps; ++sw) GCG_CUDA(cudaGraphLaunch(exec, s));
    GCG_CUDA(cudaEventRecord(ev1, s));
    k_gs_final<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), pr_old, pr_new);
    GCG_LAUNCH_CHECK();
    GCG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (out_rank) GCG_TRY(copy_out(out_rank, pr_new, (size_t)nv * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = p->max_sweeps;
        stats->converged = 0;
        stats->residual = 0.0;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = ms;
        stats->timed_sweeps = p->max_sweeps;
        stats->kernel_launches = 2 + (int)pl.nlev * p->max_sweeps;
    }
    return GCG_OK;
}

}  // namespace gcg
