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
 *
 * The same schedule runs the edge-value program of the app (PagerankProgram,
 * example_apps/pagerank.cpp:73-113, taken when num_vertices * 4 >= membudget):
 * there the value on every out-edge of u is u's pagerank / outdeg in float,
 * initially (float)(1.0/outdeg), the vertex value is the pagerank itself, and
 * each iteration logs the sum of |pagerank - old| (pagerank.cpp:108).
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

/* pagerank.cpp:80-83 (edge-value program, iteration 0): out-edges hold
 * (float)(1.0 / outdeg) */
__global__ void k_gs_edge_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float *c) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t oc = outdeg[v];
        c[v] = oc > 0 ? __double2float_rn(__ddiv_rn(1.0, (double)oc)) : 0.0f;
    }
}

/* One level of a sweep. In-memory program (EDGE = false), pagerank.cpp:127-136:
 * pr = (float)((0.15 + 0.85 * (double)sum) / outc). Edge-value program (EDGE =
 * true), pagerank.cpp:89-111: pagerank = (float)(0.15 + 0.85 * (double)sum), the
 * out-edge value pagerank / outc in float. TRACK (always with EDGE): the vertex's
 * pagerank goes to val[v] and |pagerank - previous| (float) to delta[v], for
 * the progress log and the residual stop. Levels of sweeps queued after `done`
 * was raised return at once. */
template <bool EDGE, bool TRACK>
__global__ void k_gs_level(const uint32_t *__restrict__ order, uint32_t begin, uint32_t end,
                           const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col,
                           const uint32_t *__restrict__ outdeg, const float *__restrict__ pr_old, float *pr_new,
                           float *val, float *delta, const int *done, double reset, double damping) {
    if (TRACK && *(volatile const int *)done) return;
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
        if (EDGE) pr_new[v] = outc > 0 ? __fdiv_rn(__double2float_rn(t), (float)outc) : 0.0f;
        else pr_new[v] = outc > 0 ? (float)__ddiv_rn(t, (double)outc) : (float)t;
        if (TRACK) {
            const float pagerank = __double2float_rn(t);
            delta[v] = fabsf(__fsub_rn(pagerank, val[v]));
            val[v] = pagerank;
        }
    }
}

/* The sweep's sums of delta[] and |val[]|: each block adds a fixed slice in
 * FP64, the last block to finish adds the block sums in block order, logs
 * delta_log[k] = sum delta and res_log[k] = sum delta / sum |val| for the k-th
 * sweep (k = *slot, then advanced) and raises *done when the residual is <= tol. */
constexpr int DSUM_BLOCKS = 256;
__global__ void __launch_bounds__(256) k_gs_delta_sum(const float *__restrict__ delta, const float *__restrict__ val,
                                                      uint32_t nv, double2 *part, uint32_t *ticket, uint32_t *slot,
                                                      int *done, double tol, double *delta_log, double *res_log) {
    if (*(volatile const int *)done) return;
    __shared__ double2 s[8];
    __shared__ int s_last;
    const uint32_t per = (nv + gridDim.x - 1) / gridDim.x;
    const uint32_t b0 = blockIdx.x * per, b1 = min(nv, b0 + per);
    double x = 0.0, y = 0.0;
    for (uint32_t v = b0 + threadIdx.x; v < b1; v += blockDim.x) {
        x += (double)delta[v];
        y += fabs((double)val[v]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        y += __shfl_down_sync(0xFFFFFFFFu, y, o);
    }
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = make_double2(x, y);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < 8; ++w) {
            t.x += s[w].x;
            t.y += s[w].y;
        }
        part[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    double dx = 0.0, ny = 0.0;
    for (uint32_t b = 0; b < gridDim.x; ++b) {
        const double2 p = __ldcg(part + b);
        dx += p.x;
        ny += p.y;
    }
    const uint32_t k = *slot;
    const double res = ny > 0.0 ? dx / ny : 0.0;
    delta_log[k] = dx;
    res_log[k] = res;
    *slot = k + 1;
    if (tol > 0.0 && res <= tol) *done = 1;
    *ticket = 0u;
}

/* the vertex values before the first sweep, for the progress log: the edge-value
 * program's 0.15 (pagerank.cpp:84), the in-memory program's pr * outc = 1 (or
 * 0.15 without out-edges, pagerank.cpp:137-139) */
__global__ void k_gs_val_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float reset, int edge, float *val) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        val[v] = (edge || outdeg[v] == 0) ? reset : 1.0f;
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

/* GCG_PR_GS_EXACT (in-memory program) and GCG_PR_GS_EDGE (edge-value program).
 * With tol > 0, residuals or delta_log (always for GS_EDGE) every sweep also
 * tracks the vertices' pageranks: delta_log gets sum |pagerank - previous| and
 * residuals that sum over sum |pagerank| (the Jacobi residual's definition); the
 * run stops after the first sweep whose residual is <= tol. */
int pagerank_gs_exact(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    const bool edge = p->mode == GCG_PR_GS_EDGE;
    const bool track = edge || p->tol > 0.0 || p->residuals || p->delta_log;
    GsPlan pl;
    GCG_TRY(build_gs_plan(g, pl));
    const int nsw = p->max_sweeps;
    tbuf<float> pr, val, delta;
    tbuf<double> logs; /* delta_log[nsw], res_log[nsw] */
    tbuf<double2> part;
    tbuf<uint32_t> ctl; /* ticket, slot, done */
    GCG_TRY(pr.alloc((size_t)2 * nv, s));
    GCG_TRY(ctl.alloc(4, s));
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 4 * sizeof(uint32_t), s));
    int *done = (int *)(ctl.get() + 2);
    float *pr_old = pr.get(), *pr_new = pr.get() + nv;
    const float reset = (float)p->teleport;
    if (track) {
        GCG_TRY(val.alloc(nv, s));
        GCG_TRY(delta.alloc(nv, s));
        GCG_TRY(logs.alloc(2 * (size_t)std::max(1, nsw), s));
        GCG_TRY(part.alloc(DSUM_BLOCKS, s));
        k_gs_val_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), reset, edge ? 1 : 0, val.get());
    }
    if (edge) k_gs_edge_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), pr_old);
    else k_gs_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), reset, pr_old);
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
        const unsigned gr = vgrid(e - b);
        const uint32_t *rp = g->in_rowptr.get(), *cl = g->in_col.get(), *od = g->outdeg.get();
        if (edge)
            k_gs_level<true, true><<<gr, 256, 0, cap>>>(pl.order.get(), b, e, rp, cl, od, pr_old, pr_new, val.get(),
                                                        delta.get(), done, p->teleport, p->damping);
        else if (track)
            k_gs_level<false, true><<<gr, 256, 0, cap>>>(pl.order.get(), b, e, rp, cl, od, pr_old, pr_new, val.get(),
                                                         delta.get(), done, p->teleport, p->damping);
        else
            k_gs_level<false, false><<<gr, 256, 0, cap>>>(pl.order.get(), b, e, rp, cl, od, pr_old, pr_new, nullptr,
                                                          nullptr, done, p->teleport, p->damping);
    }
    if (track)
        k_gs_delta_sum<<<DSUM_BLOCKS, 256, 0, cap>>>(delta.get(), val.get(), nv, part.get(), ctl.get(), ctl.get() + 1,
                                                     done, p->tol, logs.get(), logs.get() + std::max(1, nsw));
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
    /* sweeps are queued in chunks of 8; with a tolerance the host checks the
     * sweep count after each chunk (sweeps queued past convergence return at once) */
    uint32_t h_ctl[4] = {0, 0, 0, 0};
    GCG_CUDA(cudaEventRecord(ev0, s));
    for (int sw = 0; sw < nsw;) {
        const int n = std::min(8, nsw - sw);
        for (int k = 0; k < n; ++k) GCG_CUDA(cudaGraphLaunch(exec, s));
        sw += n;
        if (p->tol > 0.0 && sw < nsw) {
            GCG_CUDA(cudaMemcpyAsync(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            if (h_ctl[2]) break;
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaMemcpyAsync(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
    if (!edge) {
        k_gs_final<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), pr_old, pr_new);
        GCG_LAUNCH_CHECK();
    }
    GCG_CUDA(cudaEventSynchronize(ev1));
    GCG_CUDA(cudaStreamSynchronize(s));
    const int sweeps = track ? (int)h_ctl[1] : nsw;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    double last_res = 0.0;
    if (track && sweeps > 0)
        GCG_CUDA(cudaMemcpy(&last_res, logs.get() + std::max(1, nsw) + sweeps - 1, sizeof(double),
                            cudaMemcpyDeviceToHost));
    if (out_rank) GCG_TRY(copy_out(out_rank, edge ? val.get() : pr_new, (size_t)nv * 4, s));
    if (track && p->delta_log && sweeps > 0)
        GCG_TRY(copy_out(p->delta_log, logs.get(), (size_t)sweeps * sizeof(double), s));
    if (track && p->residuals && sweeps > 0)
        GCG_TRY(copy_out(p->residuals, logs.get() + std::max(1, nsw), (size_t)sweeps * sizeof(double), s));
    if (p->work_log && sweeps > 0) { /* every vertex updated per sweep; its in-edges (+ out-edges with edge values) */
        std::vector<uint64_t> wl(2 * (size_t)sweeps);
        for (int i = 0; i < sweeps; ++i) {
            wl[2 * i] = (uint64_t)nv * (uint64_t)(i + 1);
            wl[2 * i + 1] = (edge ? 2 : 1) * g->ne * (uint64_t)(i + 1);
        }
        GCG_TRY(copy_out(p->work_log, wl.data(), wl.size() * sizeof(uint64_t), s));
    }
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = (int)h_ctl[2];
        stats->residual = last_res;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = ms;
        stats->timed_sweeps = sweeps;
        stats->kernel_launches = 1 + (track ? 1 : 0) + (edge ? 0 : 1) + ((int)pl.nlev + (track ? 1 : 0)) * sweeps;
        stats->levels = (int)pl.nlev;
    }
    return GCG_OK;
}

}  // namespace gcg
