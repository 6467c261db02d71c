/*
 * PageRank on the HBM-resident in-edge CSR.
 *
 * Replaces graphchi_engine::run() driving the PageRank update()
 * (src/engine/graphchi_engine.hpp:718-992; example_apps/pagerank.cpp:73-144;
 * example_apps/pagerank_functional.cpp:48-83 with
 * src/api/functional/functional_bulksync.hpp:91-113).
 *
 * Jacobi sweep = one persistent merge-path kernel + one fix-up kernel:
 *   k_pr_sweep: per tile, gather contrib[src] for the tile's edges into shared
 *     memory, run each thread's slice of the merge path sequentially, join the
 *     slices with a block segmented scan (warp shuffles), then apply
 *     r' = (float)(teleport + damping*(double)sum), c' = r'/outdeg in float, and
 *     accumulate |r'-r| and |r'| in FP64.
 *   k_pr_fixup: finishes rows split across tiles (tail partials + head partial,
 *     in tile order) and, in the last block to finish, reduces the FP64 residual
 *     partials in a fixed order, logs the residual and raises `done` when the
 *     tolerance is met. Later sweeps already queued see `done` and return at once.
 * Algorithmic traffic per sweep: 8*E + 16*V bytes (col + gathered contrib per
 * edge; rowptr + old rank + new rank + new contrib per vertex).
 */
#include <math.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"
#include "gcg_mergepath.cuh"

namespace gcg {

namespace {

__global__ void k_plan(const uint32_t *__restrict__ rowptr, uint32_t nv, uint64_t ne, uint32_t ntiles,
                       uint32_t *__restrict__ tile_row, uint32_t *__restrict__ tile_edge) {
    const uint64_t total = (uint64_t)nv + ne;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += gridDim.x * blockDim.x) {
        uint64_t diag = (uint64_t)t * MP_TILE < total ? (uint64_t)t * MP_TILE : total;
        uint32_t r = mp_search_global(rowptr, nv, ne, diag);
        tile_row[t] = r;
        tile_edge[t] = (uint32_t)(diag - r);
    }
}

/* fix_start[t] = first tile whose tail row is the head-split row finished in t. */
__global__ void k_plan_fix(const uint32_t *__restrict__ rowptr, uint32_t ntiles, const uint32_t *__restrict__ tile_row,
                           const uint32_t *__restrict__ tile_edge, uint32_t *__restrict__ fix_start) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
        uint32_t r0 = tile_row[t];
        uint32_t res = 0xFFFFFFFFu;
        if (tile_row[t + 1] > r0 && rowptr[r0] < tile_edge[t]) {
            /* smallest k < t with tile_row[k+1] == r0 (row r0 current at the end of tile k) */
            uint32_t lo = 0, hi = t;
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (tile_row[mid + 1] >= r0) hi = mid; else lo = mid + 1;
            }
            res = lo;
        }
        fix_start[t] = res;
    }
}

struct PrArgs {
    const uint32_t *rowptr, *col, *outdeg;
    const uint32_t *tile_row, *tile_edge, *fix_start;
    uint32_t ntiles, nv;
    const float *c_old, *r_old;
    float *c_new, *r_new;
    float *head_part, *tail_part;
    double2 *block_res; /* main kernel partials (gridDim of k_pr_sweep) */
    uint32_t nblock_res;
    double2 *fix_res;   /* fix-up kernel partials */
    uint32_t *ticket;
    int *done;
    int *sweeps_done;
    double *res_log;    /* device, max_sweeps entries */
    double *last_res;
    double teleport, damping, tol;
};

__device__ __forceinline__ void pr_apply(const PrArgs &a, uint32_t v, float sum, double &dsum, double &nsum) {
    float rn = (float)(a.teleport + a.damping * (double)sum);
    float ro = a.r_old[v];
    a.r_new[v] = rn;
    uint32_t od = a.outdeg[v];
    a.c_new[v] = od ? rn / (float)od : 0.0f;
    dsum += fabs((double)rn - (double)ro);
    nsum += fabs((double)rn);
}

__device__ __forceinline__ double2 block_sum2(double a, double b, double2 *s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xFFFFFFFFu, a, o);
        b += __shfl_down_sync(0xFFFFFFFFu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_red[warp] = make_double2(a, b);
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            r.x += s_red[w].x;
            r.y += s_red[w].y;
        }
    }
    return r; /* valid in thread 0 */
}

__global__ void __launch_bounds__(MP_THREADS) k_pr_sweep(PrArgs a, int sweep) {
    if (*(volatile int *)a.done) return;
    __shared__ float s_val[MP_TILE];
    __shared__ uint32_t s_rowend[MP_TILE];
    __shared__ float s_rowsum[MP_TILE];
    __shared__ SegVal s_warp[MP_THREADS / 32];
    __shared__ double2 s_red[MP_THREADS / 32];
    const int tid = threadIdx.x;
    double dsum = 0.0, nsum = 0.0;

    for (uint32_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const uint32_t r0 = a.tile_row[t], r1 = a.tile_row[t + 1];
        const uint32_t e0 = a.tile_edge[t], e1 = a.tile_edge[t + 1];
        const uint32_t nrows = r1 - r0, nedges = e1 - e0;
        for (uint32_t k = tid; k < nrows; k += MP_THREADS) s_rowend[k] = a.rowptr[r0 + k + 1] - e0;
        for (uint32_t k = tid; k < nedges; k += MP_THREADS) s_val[k] = __ldg(a.c_old + __ldg(a.col + e0 + k));
        __syncthreads();

        const uint32_t items = nrows + nedges;
        const uint32_t d0 = min((uint32_t)tid * MP_ITEMS, items);
        const uint32_t d1 = min(d0 + MP_ITEMS, items);
        uint32_t ti = mp_search(s_rowend, nrows, nedges, d0);
        uint32_t tj = d0 - ti;
        float run = 0.0f, first_part = 0.0f;
        int first_row = -1;
        for (uint32_t d = d0; d < d1; ++d) {
            if (ti < nrows && s_rowend[ti] <= tj) {
                if (first_row < 0) {
                    first_row = (int)ti;
                    first_part = run;
                } else {
                    s_rowsum[ti] = run;
                }
                run = 0.0f;
                ++ti;
            } else {
                run += s_val[tj];
                ++tj;
            }
        }
        float tile_tail;
        float carry = seg_scan_excl(SegVal{first_row >= 0 ? 1 : 0, run}, s_warp, &tile_tail);
        if (first_row >= 0) s_rowsum[first_row] = carry + first_part;
        __syncthreads();
        const bool head_split = a.rowptr[r0] < e0;
        if (tid == 0) {
            a.tail_part[t] = tile_tail;
            if (head_split && nrows > 0) a.head_part[t] = s_rowsum[0];
        }
        for (uint32_t k = tid; k < nrows; k += MP_THREADS) {
            if (k == 0 && head_split) continue;
            pr_apply(a, r0 + k, s_rowsum[k], dsum, nsum);
        }
        __syncthreads();
    }
    double2 r = block_sum2(dsum, nsum, s_red);
    if (tid == 0) a.block_res[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) k_pr_fixup(PrArgs a, int sweep) {
    if (*(volatile int *)a.done) return;
    __shared__ double2 s_red[8];
    __shared__ int s_last;
    double dsum = 0.0, nsum = 0.0;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ntiles; t += gridDim.x * blockDim.x) {
        uint32_t ts = a.fix_start[t];
        if (ts == 0xFFFFFFFFu) continue;
        float sum = a.tail_part[ts];
        for (uint32_t k = ts + 1; k < t; ++k) sum += a.tail_part[k];
        sum += a.head_part[t];
        pr_apply(a, a.tile_row[t], sum, dsum, nsum);
    }
    double2 r = block_sum2(dsum, nsum, s_red);
    if (threadIdx.x == 0) {
        a.fix_res[blockIdx.x] = r;
        __threadfence();
        unsigned prev = atomicAdd(a.ticket, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    /* last block: fixed-order reduction of all partials */
    double x = 0.0, y = 0.0;
    for (uint32_t i = threadIdx.x; i < a.nblock_res; i += blockDim.x) {
        double2 p = __ldcg(a.block_res + i);
        x += p.x;
        y += p.y;
    }
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        double2 p = __ldcg(a.fix_res + i);
        x += p.x;
        y += p.y;
    }
    __syncthreads();
    double2 tot = block_sum2(x, y, s_red);
    if (threadIdx.x == 0) {
        double res = tot.y > 0.0 ? tot.x / tot.y : 0.0;
        a.res_log[sweep] = res;
        *a.last_res = res;
        *a.sweeps_done = sweep + 1;
        if (a.tol > 0.0 && res <= a.tol) *a.done = 1;
        *a.ticket = 0u;
    }
}

__global__ void k_pr_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float init, const float *__restrict__ init_rank,
                          float *__restrict__ r, float *__restrict__ c) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        float x = init_rank ? init_rank[v] : init;
        r[v] = x;
        uint32_t od = outdeg[v];
        c[v] = od ? x / (float)od : 0.0f;
    }
}

}  // namespace

int ensure_plan(gcg_graph *g) {
    if (g->plan) return GCG_OK;
    PrPlan *p = new PrPlan();
    const uint64_t total = (uint64_t)g->nv + g->ne;
    p->ntiles = (uint32_t)((total + MP_TILE - 1) / MP_TILE);
    if (p->tile_row.alloc((size_t)p->ntiles + 1) || p->tile_edge.alloc((size_t)p->ntiles + 1) ||
        p->fix_start.alloc((size_t)p->ntiles + 1)) {
        delete p;
        return GCG_ERR_NOMEM;
    }
    unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)p->ntiles + 256) / 256, 4096));
    k_plan<<<blocks, 256, 0, g->stream>>>(g->in_rowptr.get(), g->nv, g->ne, p->ntiles, p->tile_row.get(),
                                          p->tile_edge.get());
    k_plan_fix<<<blocks, 256, 0, g->stream>>>(g->in_rowptr.get(), p->ntiles, p->tile_row.get(), p->tile_edge.get(),
                                              p->fix_start.get());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        delete p;
        return fail(GCG_ERR_CUDA, std::string("merge-path plan: ") + cudaGetErrorString(e));
    }
    g->plan = p;
    return GCG_OK;
}

static int sweep_grid(uint32_t ntiles) {
    static int per_sm = 0;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_sweep, MP_THREADS, 0) != cudaSuccess ||
            per_sm <= 0) {
            cudaGetLastError();
            per_sm = 4;
        }
    }
    int g = num_sms() * per_sm;
    if ((uint32_t)g > ntiles) g = (int)std::max<uint32_t>(ntiles, 1);
    return g;
}

static int pagerank_jacobi(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    GCG_TRY(ensure_plan(g));
    cudaStream_t s = g->stream;
    const PrPlan &pl = *g->plan;
    const uint32_t nv = g->nv;
    const int max_sweeps = p->max_sweeps;

    tbuf<float> r, c, parts;
    tbuf<double2> bres, fres;
    tbuf<uint32_t> ctl;   /* ticket, done, sweeps_done */
    tbuf<double> dres;    /* res_log[max_sweeps] + last_res */
    const int g1 = sweep_grid(pl.ntiles);
    const int g2 = (int)std::max<uint32_t>(1, std::min<uint32_t>((pl.ntiles + 255) / 256, (uint32_t)num_sms() * 4));
    GCG_TRY(r.alloc((size_t)2 * nv, s));
    GCG_TRY(c.alloc((size_t)2 * nv, s));
    GCG_TRY(parts.alloc((size_t)2 * pl.ntiles + 2, s));
    GCG_TRY(bres.alloc(g1, s));
    GCG_TRY(fres.alloc(g2, s));
    GCG_TRY(ctl.alloc(4, s));
    GCG_TRY(dres.alloc((size_t)max_sweeps + 1, s));
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 4 * sizeof(uint32_t), s));
    GCG_CUDA(cudaMemsetAsync(dres.get(), 0, ((size_t)max_sweeps + 1) * sizeof(double), s));

    /* initial vector: caller's (warm start) or the constant init */
    tbuf<float> init_stage;
    const float *init_dev = nullptr;
    if (p->init_rank) {
        if (is_device_ptr(p->init_rank)) {
            init_dev = p->init_rank;
        } else {
            GCG_TRY(init_stage.alloc(nv, s));
            GCG_TRY(copy_in(init_stage.get(), p->init_rank, (size_t)nv * 4, s));
            init_dev = init_stage.get();
        }
    }
    unsigned vb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, (uint64_t)num_sms() * 8));
    k_pr_init<<<vb, 256, 0, s>>>(nv, g->outdeg.get(), p->init, init_dev, r.get(), c.get());
    GCG_LAUNCH_CHECK();

    PrArgs a;
    a.rowptr = g->in_rowptr.get();
    a.col = g->in_col.get();
    a.outdeg = g->outdeg.get();
    a.tile_row = pl.tile_row.get();
    a.tile_edge = pl.tile_edge.get();
    a.fix_start = pl.fix_start.get();
    a.ntiles = pl.ntiles;
    a.nv = nv;
    a.head_part = parts.get();
    a.tail_part = parts.get() + pl.ntiles + 1;
    a.block_res = bres.get();
    a.nblock_res = (uint32_t)g1;
    a.fix_res = fres.get();
    a.ticket = ctl.get();
    a.done = (int *)(ctl.get() + 1);
    a.sweeps_done = (int *)(ctl.get() + 2);
    a.res_log = dres.get();
    a.last_res = dres.get() + max_sweeps;
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.tol = p->tol;

    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    const bool time_sweeps = (p->flags & GCG_PR_TIME_SWEEPS) != 0;
    std::vector<cudaEvent_t> sweep_ev; /* pairs around each main sweep kernel */

    /* Sweeps are queued in chunks; after each chunk the done flag is copied to
     * pinned memory. The host waits on the chunk before last, so the GPU always
     * has work queued; sweeps queued past convergence return immediately. */
    const int CHUNK = 4;
    int *h_flags = nullptr;
    GCG_CUDA(cudaMallocHost((void **)&h_flags, 64 * sizeof(int)));
    std::vector<cudaEvent_t> chunk_ev;
    int launched = 0, stop = 0;
    int status = GCG_OK;
    while (launched < max_sweeps && !stop) {
        int n = std::min(CHUNK, max_sweeps - launched);
        for (int k = 0; k < n; ++k) {
            const int sw = launched + k;
            a.r_old = r.get() + (size_t)(sw & 1) * nv;
            a.c_old = c.get() + (size_t)(sw & 1) * nv;
            a.r_new = r.get() + (size_t)((sw + 1) & 1) * nv;
            a.c_new = c.get() + (size_t)((sw + 1) & 1) * nv;
            if (time_sweeps) {
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, s);
                k_pr_sweep<<<g1, MP_THREADS, 0, s>>>(a, sw);
                cudaEventRecord(e1, s);
                sweep_ev.push_back(e0);
                sweep_ev.push_back(e1);
            } else {
                k_pr_sweep<<<g1, MP_THREADS, 0, s>>>(a, sw);
            }
            k_pr_fixup<<<g2, 256, 0, s>>>(a, sw);
        }
        launched += n;
        if (cudaGetLastError() != cudaSuccess) {
            status = fail(GCG_ERR_CUDA, "pagerank sweep launch failed");
            break;
        }
        if (p->tol > 0.0) {
            int slot = (int)chunk_ev.size() % 64;
            cudaMemcpyAsync(h_flags + slot, a.done, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaEvent_t e;
            cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            cudaEventRecord(e, s);
            chunk_ev.push_back(e);
            /* wait for the previous chunk's flag */
            if (chunk_ev.size() >= 2) {
                size_t idx = chunk_ev.size() - 2;
                cudaEventSynchronize(chunk_ev[idx]);
                if (h_flags[idx % 64]) stop = 1;
            }
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaEventSynchronize(ev1));
    for (auto e : chunk_ev) cudaEventDestroy(e);
    cudaFreeHost(h_flags);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (status != GCG_OK) {
        for (auto e : sweep_ev) cudaEventDestroy(e);
        return status;
    }

    uint32_t h_ctl[4];
    GCG_CUDA(cudaMemcpy(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost));
    const int sweeps = (int)h_ctl[2];
    const int done = (int)h_ctl[1];
    double sweep_ms = 0.0;
    int timed = 0;
    for (size_t i = 0; i + 1 < sweep_ev.size(); i += 2) {
        if ((int)(i / 2) < sweeps) { /* launches after convergence returned at once: not counted */
            float t = 0.0f;
            cudaEventElapsedTime(&t, sweep_ev[i], sweep_ev[i + 1]);
            sweep_ms += t;
            ++timed;
        }
        cudaEventDestroy(sweep_ev[i]);
        cudaEventDestroy(sweep_ev[i + 1]);
    }
    double last_res = 0.0;
    GCG_CUDA(cudaMemcpy(&last_res, a.last_res, sizeof(double), cudaMemcpyDeviceToHost));
    if (p->residuals && sweeps > 0) GCG_TRY(copy_out(p->residuals, dres.get(), (size_t)sweeps * sizeof(double), s));
    const float *result = r.get() + (size_t)(sweeps & 1) * nv;
    if (out_rank) GCG_TRY(copy_out(out_rank, result, (size_t)nv * sizeof(float), s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = done;
        stats->residual = last_res;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = sweep_ms;
        stats->timed_sweeps = timed;
        stats->kernel_launches = 1 + 2 * launched;
    }
    return GCG_OK;
}

}  // namespace gcg

using namespace gcg;

extern "C" {

void gcg_pr_params_default(gcg_pr_params *p) {
    if (!p) return;
    p->mode = GCG_PR_JACOBI;
    p->max_sweeps = 3;
    p->teleport = 0.15;
    p->damping = 0.85;
    p->tol = 0.0;
    p->init = 1.0f;
    p->flags = 0u;
    p->init_rank = nullptr;
    p->residuals = nullptr;
}

int gcg_pagerank(gcg_graph *g, const gcg_pr_params *params, float *out_rank, gcg_pr_stats *stats) {
    if (!g || !params) return fail(GCG_ERR_INVALID, "gcg_pagerank: null argument");
    if (params->max_sweeps < 0) return fail(GCG_ERR_INVALID, "gcg_pagerank: max_sweeps < 0");
    if (params->mode == GCG_PR_JACOBI) return pagerank_jacobi(g, params, out_rank, stats);
    if (params->mode == GCG_PR_GS_EXACT) return pagerank_gs_exact(g, params, out_rank, stats);
    return fail(GCG_ERR_INVALID, "gcg_pagerank: unknown mode");
}

}  // extern "C"
