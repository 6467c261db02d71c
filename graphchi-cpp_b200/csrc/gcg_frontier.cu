/*
 * Selective scheduling as a device frontier, and the two programs that use it.
 *
 * The reference's bitset_scheduler (src/engine/bitset_scheduler.hpp:38-104) keeps
 * two dense bitsets: add_task sets a vertex's bit for the next iteration,
 * new_iteration swaps the two and clears the new "next", is_scheduled reads the
 * current one, and the engine stops when an iteration scheduled nothing
 * (graphchi_engine.hpp:477-501, 801-814). Here the two bitsets live in HBM
 * (one bit per vertex, 32-bit words, atomicOr to schedule); at the start of an
 * iteration the current bitset is compacted into a vertex list (per-word
 * popcounts, an exclusive scan, a scatter), so the iteration's kernels run over
 * scheduled vertices only, a warp per vertex.
 *
 * Programs:
 *   CC by label propagation (example_apps/connectedcomponents.cpp:79-138): in
 *   iteration 0 every vertex takes the minimum of its id and its neighbours' ids;
 *   afterwards a vertex takes the minimum label over its neighbourhood. Without
 *   the scheduler every vertex is updated every iteration (Jacobi, double
 *   buffered); with it, a vertex whose label dropped schedules its neighbours
 *   (push: atomicMin into each neighbour, which is scheduled when its label
 *   dropped). Both stop at the fixpoint: the minimum id per weak component,
 *   the same labels as gcg_connected_components.
 *   Delta PageRank (GCG_PR_DELTA): Jacobi sweeps over the scheduled vertices
 *   only; sweep 0 schedules all; a vertex whose rank moved by more than
 *   delta_threshold x its new rank schedules its out-neighbours. With threshold
 *   0 every change propagates and the sweeps equal plain Jacobi sweeps.
 */
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

/* ---- the frontier --------------------------------------------------------- */

__global__ void k_bits_all(uint32_t *bits, uint32_t nv) {
    const uint32_t nw = (nv + 31) / 32;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        const uint32_t rem = nv - w * 32;
        bits[w] = rem >= 32 ? 0xFFFFFFFFu : ((1u << rem) - 1u);
    }
}

__global__ void k_bits_popc(const uint32_t *__restrict__ bits, uint32_t nw, uint32_t *__restrict__ cnt) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x)
        cnt[w] = __popc(bits[w]);
}

__global__ void k_bits_scatter(const uint32_t *__restrict__ bits, uint32_t nw, const uint32_t *__restrict__ off,
                               uint32_t *__restrict__ list) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        uint32_t b = bits[w], o = off[w];
        while (b) {
            const int i = __ffs(b) - 1;
            b &= b - 1;
            list[o++] = w * 32 + (uint32_t)i;
        }
    }
}

__device__ __forceinline__ void schedule(uint32_t *bits, uint32_t v) {
    const uint32_t m = 1u << (v & 31u);
    if (!(((volatile uint32_t *)bits)[v >> 5] & m)) atomicOr(bits + (v >> 5), m);
}

/* neighbourhood: in-list ++ out-list (rout NULL: the in-list is the whole of it) */
struct Nb {
    const uint32_t *rin, *cin, *rout, *cout;
};
__device__ __forceinline__ uint32_t nb_count(const Nb &n, uint32_t v) {
    uint32_t d = n.rin[v + 1] - n.rin[v];
    if (n.rout) d += n.rout[v + 1] - n.rout[v];
    return d;
}
__device__ __forceinline__ uint32_t nb_at(const Nb &n, uint32_t v, uint32_t i) {
    const uint32_t b = n.rin[v], din = n.rin[v + 1] - b;
    return i < din ? n.cin[b + i] : n.cout[n.rout[v] + (i - din)];
}

/* ---- CC by label propagation ------------------------------------------------ */

/* Jacobi step over all vertices: lab_new[v] = min(lab[v], min over neighbours);
 * iteration 0 reads neighbour ids (connectedcomponents.cpp:93-94). *changed
 * counts the vertices whose label dropped. */
__global__ void k_lp_pull(Nb n, uint32_t nv, int first, const uint32_t *__restrict__ lab, uint32_t *__restrict__ lab_new,
                          unsigned long long *changed) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long ch = 0;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarps) {
        const uint32_t d = nb_count(n, v);
        const uint32_t own = first ? v : lab[v];
        uint32_t m = own;
        for (uint32_t i = lane; i < d; i += 32u) {
            const uint32_t u = nb_at(n, v, i);
            m = min(m, first ? u : lab[u]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
        if (lane == 0) {
            lab_new[v] = m;
            ch += m < own;
        }
    }
    if (lane == 0 && ch) atomicAdd(changed, ch);
}

__global__ void k_lp_init(uint32_t *lab, uint32_t nv) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) lab[v] = v;
}

/* scheduled step: every listed vertex pushes its label into its neighbours; a
 * neighbour whose label dropped is scheduled for the next iteration */
__global__ void k_lp_push(Nb n, const uint32_t *__restrict__ list, uint32_t count, uint32_t *lab, uint32_t *next,
                          unsigned long long *work) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long wk = 0;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < count; k += nwarps) {
        const uint32_t v = list[k], d = nb_count(n, v);
        const uint32_t l = ((volatile uint32_t *)lab)[v];
        for (uint32_t i = lane; i < d; i += 32u) {
            const uint32_t u = nb_at(n, v, i);
            if (((volatile uint32_t *)lab)[u] > l && atomicMin(lab + u, l) > l) schedule(next, u);
        }
        wk += d;
    }
    if (lane == 0 && wk) atomicAdd(work, wk);
}

/* ---- delta PageRank ----------------------------------------------------- */

struct DeltaArgs {
    const uint32_t *rin, *cin, *rout, *cout, *outdeg;
    const uint32_t *list;
    uint32_t count;
    float *r;            /* ranks (each vertex writes only its own) */
    const float *c;      /* contributions of the sweep's start */
    float *c_next;       /* contributions written by this sweep's vertices */
    uint32_t *next;      /* next iteration's bitset */
    double teleport, damping, threshold;
    double2 *part;       /* per block b: [2b] = (sum |r' - r|, sum |r'|), [2b+1] = (sum |r|, 0) over its vertices */
    unsigned long long *work;
};

/* a warp per scheduled vertex: the in-edge sum in a fixed order (lane-strided
 * partial sums, then a fixed xor tree), the apply formula of the Jacobi path,
 * and the scheduling of the out-neighbours when the change is above threshold */
__global__ void __launch_bounds__(256) k_delta_sweep(DeltaArgs a) {
    __shared__ double s_p[8][3];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double dsum = 0.0, nsum = 0.0, osum = 0.0;
    unsigned long long wk = 0;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < a.count; k += nwarps) {
        const uint32_t v = a.list[k];
        const uint32_t b = a.rin[v], e = a.rin[v + 1];
        float s = 0.0f;
        for (uint32_t i = b + lane; i < e; i += 32u) s += a.c[a.cin[i]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        const float rn = (float)__dadd_rn(a.teleport, __dmul_rn(a.damping, (double)s));
        const float ro = a.r[v];
        const uint32_t od = a.outdeg[v];
        const double dr = fabs((double)rn - (double)ro);
        if (lane == 0) {
            a.r[v] = rn;
            a.c_next[v] = od ? __fdiv_rn(rn, (float)od) : 0.0f;
            dsum += dr;
            nsum += fabs((double)rn);
            osum += fabs((double)ro);
            wk += e - b;
        }
        if (dr > a.threshold * fabs((double)rn)) {
            const uint32_t ob = a.rout[v], oe = a.rout[v + 1];
            for (uint32_t i = ob + lane; i < oe; i += 32u) schedule(a.next, a.cout[i]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dsum += __shfl_xor_sync(FULL, dsum, o);
        nsum += __shfl_xor_sync(FULL, nsum, o);
        osum += __shfl_xor_sync(FULL, osum, o);
    }
    if (lane == 0) {
        s_p[warp][0] = dsum;
        s_p[warp][1] = nsum;
        s_p[warp][2] = osum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t0 += s_p[w][0];
            t1 += s_p[w][1];
            t2 += s_p[w][2];
        }
        a.part[2 * blockIdx.x] = make_double2(t0, t1);
        a.part[2 * blockIdx.x + 1] = make_double2(t2, 0.0);
    }
    if (lane == 0 && wk) atomicAdd(a.work, wk);
}

/* after the sweep: the updated vertices' new contributions become current */
__global__ void k_delta_commit(const uint32_t *__restrict__ list, uint32_t count, const float *__restrict__ c_next,
                               float *__restrict__ c) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t v = list[k];
        c[v] = c_next[v];
    }
}

__global__ void k_delta_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float init, const float *init_rank,
                             float *__restrict__ r, float *__restrict__ c) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const float x = init_rank ? init_rank[v] : init;
        const uint32_t od = outdeg[v];
        r[v] = x;
        c[v] = od ? __fdiv_rn(x, (float)od) : 0.0f;
    }
}

unsigned grid_for(uint64_t n, unsigned per = 256, unsigned mult = 8) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + per - 1) / per, (uint64_t)num_sms() * mult));
}

/* the current bitset -> a vertex list; returns the count (host) */
int compact(const uint32_t *bits, uint32_t nv, uint32_t *cnt, uint32_t *list, uint32_t *total, cudaStream_t s,
            uint32_t *count) {
    const uint32_t nw = (nv + 31) / 32;
    k_bits_popc<<<grid_for(nw), 256, 0, s>>>(bits, nw, cnt);
    GCG_TRY(scan_u32(cnt, cnt, nw, total, s));
    k_bits_scatter<<<grid_for(nw), 256, 0, s>>>(bits, nw, cnt, list);
    GCG_LAUNCH_CHECK();
    GCG_CUDA(cudaMemcpyAsync(count, total, 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

}  // namespace

/* ---- host drivers ----------------------------------------------------------- */

int cc_label_propagation(gcg_graph *g, int scheduler, int max_iters, uint32_t *labels, gcg_cc_stats *stats,
                         int32_t *frontier_log) {
    if (!g->symmetric && !g->has_out)
        return fail(GCG_ERR_UNSUPPORTED,
                    "label propagation needs whole neighbourhoods: build the graph with GCG_BUILD_SYMMETRISE or with "
                    "its out-edge CSR");
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv, nw = (nv + 31) / 32;
    Nb n;
    n.rin = g->in_rowptr.get();
    n.cin = g->in_col.get();
    n.rout = g->symmetric ? nullptr : g->out_rowptr.get();
    n.cout = g->symmetric ? nullptr : g->out_col.get();
    tbuf<uint32_t> lab, lab2, bits, cnt, list, total;
    tbuf<unsigned long long> ctr;
    GCG_TRY(lab.alloc(nv, s));
    GCG_TRY(ctr.alloc(2, s));
    const bool dev_out = labels && is_device_ptr(labels);
    std::vector<int32_t> flog;
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    int iters = 0;
    uint32_t *cur = lab.get();
    if (!scheduler) {
        GCG_TRY(lab2.alloc(nv, s));
        uint32_t *nxt = lab2.get();
        for (int it = 0; it < max_iters; ++it) {
            GCG_CUDA(cudaMemsetAsync(ctr.get(), 0, 8, s));
            k_lp_pull<<<grid_for((uint64_t)nv * 32, 256, 16), 256, 0, s>>>(n, nv, it == 0, cur, nxt, ctr.get());
            GCG_LAUNCH_CHECK();
            unsigned long long changed = 0;
            GCG_CUDA(cudaMemcpyAsync(&changed, ctr.get(), 8, cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            std::swap(cur, nxt);
            ++iters;
            flog.push_back((int32_t)nv);
            if (changed == 0 && it > 0) break; /* the fixpoint (connectedcomponents.cpp:125-138) */
        }
    } else {
        /* iteration 0 schedules every vertex (add_task_to_all); a push of the
         * initial labels (ids) is the reference's iteration 0 */
        GCG_TRY(bits.alloc((size_t)2 * std::max<uint32_t>(nw, 1), s));
        GCG_TRY(cnt.alloc(std::max<uint32_t>(nw, 1), s));
        GCG_TRY(list.alloc(std::max<uint32_t>(nv, 1), s));
        GCG_TRY(total.alloc(1, s));
        uint32_t *bc = bits.get(), *bn = bits.get() + std::max<uint32_t>(nw, 1);
        k_lp_init<<<grid_for(nv), 256, 0, s>>>(cur, nv);
        k_bits_all<<<grid_for(nw), 256, 0, s>>>(bc, nv);
        GCG_CUDA(cudaMemsetAsync(bn, 0, (size_t)nw * 4, s));
        GCG_CUDA(cudaMemsetAsync(ctr.get(), 0, 16, s));
        for (int it = 0; it < max_iters; ++it) {
            uint32_t count = 0;
            GCG_TRY(compact(bc, nv, cnt.get(), list.get(), total.get(), s, &count));
            if (count == 0) break; /* nothing scheduled: has_new_tasks is false */
            k_lp_push<<<grid_for((uint64_t)count * 32, 256, 16), 256, 0, s>>>(n, list.get(), count, cur, bn,
                                                                              ctr.get() + 1);
            GCG_LAUNCH_CHECK();
            flog.push_back((int32_t)count);
            ++iters;
            std::swap(bc, bn); /* new_iteration: swap, clear the new next */
            GCG_CUDA(cudaMemsetAsync(bn, 0, (size_t)nw * 4, s));
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    /* components: vertices that are their own label */
    std::vector<uint32_t> h(nv);
    GCG_CUDA(cudaMemcpyAsync(h.data(), cur, (size_t)nv * 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (labels) GCG_CUDA(cudaMemcpy(labels, dev_out ? (const void *)cur : (const void *)h.data(), (size_t)nv * 4,
                                    cudaMemcpyDefault));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (frontier_log && !flog.empty()) GCG_TRY(copy_out(frontier_log, flog.data(), flog.size() * 4, s));
    if (stats) {
        uint32_t roots = 0;
        for (uint32_t v = 0; v < nv; ++v) roots += h[v] == v;
        stats->passes = iters;
        stats->ncomponents = roots;
        stats->device_ms = ms;
    }
    return GCG_OK;
}

int pagerank_delta(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    if (!g->has_out)
        return fail(GCG_ERR_UNSUPPORTED, "GCG_PR_DELTA schedules out-neighbours: build the graph with its out-edge CSR");
    if (!(p->delta_threshold >= 0.0)) return fail(GCG_ERR_INVALID, "gcg_pagerank: delta_threshold must be >= 0");
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv, nw = (nv + 31) / 32;
    const int max_sweeps = p->max_sweeps;
    tbuf<float> r, c, cn, init_stage;
    tbuf<uint32_t> bits, cnt, list, total;
    tbuf<double2> part;
    tbuf<unsigned long long> work;
    const unsigned sb = (unsigned)(num_sms() * 8);
    GCG_TRY(r.alloc(nv, s));
    GCG_TRY(c.alloc(nv, s));
    GCG_TRY(cn.alloc(nv, s));
    GCG_TRY(bits.alloc((size_t)2 * std::max<uint32_t>(nw, 1), s));
    GCG_TRY(cnt.alloc(std::max<uint32_t>(nw, 1), s));
    GCG_TRY(list.alloc(std::max<uint32_t>(nv, 1), s));
    GCG_TRY(total.alloc(1, s));
    GCG_TRY(part.alloc(2 * (size_t)sb, s));
    GCG_TRY(work.alloc(1, s));
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
    uint32_t *bc = bits.get(), *bn = bits.get() + std::max<uint32_t>(nw, 1);
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    k_delta_init<<<grid_for(nv), 256, 0, s>>>(nv, g->outdeg.get(), p->init, init_dev, r.get(), c.get());
    k_bits_all<<<grid_for(nw), 256, 0, s>>>(bc, nv);
    GCG_CUDA(cudaMemsetAsync(bn, 0, (size_t)nw * 4, s));
    GCG_CUDA(cudaMemsetAsync(work.get(), 0, 8, s));
    DeltaArgs a;
    a.rin = g->in_rowptr.get();
    a.cin = g->in_col.get();
    a.rout = g->out_rowptr.get();
    a.cout = g->out_col.get();
    a.outdeg = g->outdeg.get();
    a.r = r.get();
    a.c = c.get();
    a.c_next = cn.get();
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.threshold = p->delta_threshold;
    a.part = part.get();
    a.work = work.get();
    std::vector<double> res_log, delta_log;
    std::vector<uint64_t> work_log;
    std::vector<double2> hp(2 * (size_t)sb);
    uint64_t nupdates = 0;
    int sweeps = 0, launches = 3;
    double last = 0.0;
    double total_rank = 0.0; /* sum of |r| over all vertices, kept current from the updated ones */
    for (int it = 0; it < max_sweeps; ++it) {
        uint32_t count = 0;
        GCG_TRY(compact(bc, nv, cnt.get(), list.get(), total.get(), s, &count));
        launches += 2;
        if (count == 0) break;
        a.list = list.get();
        a.count = count;
        a.next = bn;
        const unsigned gb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)count * 32 + 255) / 256, sb));
        k_delta_sweep<<<gb, 256, 0, s>>>(a);
        k_delta_commit<<<grid_for(count), 256, 0, s>>>(list.get(), count, cn.get(), c.get());
        GCG_LAUNCH_CHECK();
        launches += 2;
        unsigned long long wk = 0;
        GCG_CUDA(cudaMemcpyAsync(hp.data(), part.get(), 2 * (size_t)gb * sizeof(double2), cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaMemcpyAsync(&wk, work.get(), 8, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        double d = 0.0, nrm = 0.0, old = 0.0;
        for (unsigned b = 0; b < gb; ++b) { /* fixed order */
            d += hp[2 * b].x;
            nrm += hp[2 * b].y;
            old += hp[2 * b + 1].x;
        }
        /* the whole vector's L1 norm after the sweep: every vertex is in sweep 0,
         * later sweeps change only the updated ones */
        total_rank = it == 0 ? nrm : total_rank + (nrm - old);
        last = total_rank > 0.0 ? d / total_rank : 0.0; /* normalised L1 change of the whole vector */
        res_log.push_back(last);
        delta_log.push_back(d);
        nupdates += count;
        work_log.push_back(nupdates);
        work_log.push_back(wk);
        ++sweeps;
        std::swap(bc, bn); /* new_iteration */
        GCG_CUDA(cudaMemsetAsync(bn, 0, (size_t)nw * 4, s));
        if (p->tol > 0.0 && last <= p->tol) break;
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (out_rank) GCG_TRY(copy_out(out_rank, r.get(), (size_t)nv * 4, s));
    if (p->residuals && sweeps) GCG_TRY(copy_out(p->residuals, res_log.data(), res_log.size() * 8, s));
    if (p->delta_log && sweeps) GCG_TRY(copy_out(p->delta_log, delta_log.data(), delta_log.size() * 8, s));
    if (p->work_log && sweeps) GCG_TRY(copy_out(p->work_log, work_log.data(), work_log.size() * 8, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = (p->tol > 0.0 && last <= p->tol) || (sweeps < max_sweeps);
        stats->residual = last;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = 0.0;
        stats->timed_sweeps = 0;
        stats->kernel_launches = launches;
    }
    return GCG_OK;
}

}  // namespace gcg
