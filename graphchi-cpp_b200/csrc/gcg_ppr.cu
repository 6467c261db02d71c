/*
 * Batched personalised PageRank: k sources at once as a dense rank matrix.
 *
 * No reference counterpart (the reference runs one vector per engine run,
 * example_apps/pagerank.cpp); the per-source semantics are those of the
 * personalised scalar path: r_s[v] = (float)(tele_s(v) + damping*(double)sum_{u->v}
 * c_s[u]) with tele_s(v) = teleport if v == source_s else 0, c_s[u] = r_s[u]/outdeg[u]
 * in float, r_s starting at the indicator of source_s, and a stop when the largest
 * per-source normalised L1 change (FP64) is <= tol.
 *
 * Layout: vertex-major matrices R[V][kp], C[V][kp] (kp = k rounded up to 32, at most
 * 256 per group; larger k run group by group), so the contribution row of a source
 * vertex is one contiguous 4*kp-byte line: a warp gathers it with one 128-bit load
 * per lane per 32 columns (fully coalesced, 1 KiB per edge at kp = 256).
 * Work: in-edge rows are cut into segments of at most 256 edges; one warp per
 * segment broadcasts the segment's source ids with shuffles, keeps four row
 * gathers in flight, and accumulates in registers (lane = 8 columns). A row of one
 * segment is applied at once; longer rows leave per-segment partials that a
 * fix-up pass adds in segment order. Vertices without in-edges are constant after
 * the first sweep and are written only in sweeps 0 and 1. Per-column FP64
 * residuals are reduced in a fixed order.
 * Algorithmic traffic per sweep: E*(4 + 4*kp) + 3*V*4*kp bytes.
 */
#include <math.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

constexpr uint32_t SEG = 256;     /* edges per segment */
constexpr int PPR_THREADS = 256;  /* 8 warps */
constexpr uint32_t KMAX = 256;    /* columns per group */
constexpr uint32_t NONE = 0xFFFFFFFFu;

template <int CPL>
__device__ __forceinline__ void load_row(const float *p, float (&x)[CPL]) {
    if constexpr (CPL == 8) {
        const float4 a = __ldg((const float4 *)p), b = __ldg((const float4 *)p + 1);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    } else if constexpr (CPL == 4) {
        const float4 a = __ldg((const float4 *)p);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    } else if constexpr (CPL == 2) {
        const float2 a = __ldg((const float2 *)p);
        x[0] = a.x; x[1] = a.y;
    } else {
        x[0] = __ldg(p);
    }
}

template <int CPL>
__device__ __forceinline__ void store_row(float *p, const float (&x)[CPL]) {
    if constexpr (CPL == 8) {
        ((float4 *)p)[0] = make_float4(x[0], x[1], x[2], x[3]);
        ((float4 *)p)[1] = make_float4(x[4], x[5], x[6], x[7]);
    } else if constexpr (CPL == 4) {
        ((float4 *)p)[0] = make_float4(x[0], x[1], x[2], x[3]);
    } else if constexpr (CPL == 2) {
        ((float2 *)p)[0] = make_float2(x[0], x[1]);
    } else {
        p[0] = x[0];
    }
}

struct PprArgs {
    const uint32_t *col, *outdeg;
    const uint4 *seg;        /* (row, edge begin, edge end, partial slot or NONE) */
    const uint4 *multi;      /* (row, first slot, segment count, 0) */
    const uint32_t *zero_rows;
    uint32_t nseg, nmulti, nzero, kp, k;
    const uint32_t *src;     /* kp source ids (NONE for padding columns) */
    const float *c_old, *r_old;
    float *c_new, *r_new, *partial;
    double2 *bpart;          /* per block, per column (|dr|, |r|) */
    uint32_t nbseg;          /* blocks of the segment kernel (their partials come first) */
    uint32_t *ticket;
    int *done, *sweeps_done;
    double *res_log, *last_res;
    const double *norm_const; /* per column: |r| of constant vertices once no longer visited */
    double teleport, damping, tol;
};

/* apply one row: r' = tele + damping*sum, c' = r'/outdeg, residual per column */
template <int CPL>
__device__ __forceinline__ void ppr_apply(const PprArgs &a, uint32_t v, const float (&sum)[CPL], const uint32_t (&srcs)[CPL],
                                          uint32_t lane, double (&dsum)[CPL], double (&nsum)[CPL]) {
    const size_t off = (size_t)v * a.kp + (size_t)lane * CPL;
    float ro[CPL], rn[CPL], cn[CPL];
    load_row<CPL>(a.r_old + off, ro);
    const uint32_t od = a.outdeg[v];
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
        const double tele = srcs[j] == v ? a.teleport : 0.0;
        rn[j] = (float)__dadd_rn(tele, __dmul_rn(a.damping, (double)sum[j]));
        cn[j] = od ? __fdiv_rn(rn[j], (float)od) : 0.0f;
        dsum[j] += fabs((double)rn[j] - (double)ro[j]);
        nsum[j] += fabs((double)rn[j]);
    }
    store_row<CPL>(a.r_new + off, rn);
    store_row<CPL>(a.c_new + off, cn);
}

/* block-level fixed-order reduction of the per-lane column residuals */
template <int CPL>
__device__ __forceinline__ void block_columns(const PprArgs &a, double (&dsum)[CPL], double (&nsum)[CPL],
                                              double2 *s_part, uint32_t out_block) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < CPL; ++j) s_part[warp * KMAX + lane * CPL + j] = make_double2(dsum[j], nsum[j]);
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < a.kp; c += blockDim.x) {
        double2 t = make_double2(0.0, 0.0);
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
            t.x += s_part[w * KMAX + c].x;
            t.y += s_part[w * KMAX + c].y;
        }
        a.bpart[(size_t)out_block * a.kp + c] = t;
    }
}

template <int CPL>
__global__ void __launch_bounds__(PPR_THREADS) k_ppr_seg(PprArgs a) {
    if (*(volatile const int *)a.done) return;
    __shared__ double2 s_part[(PPR_THREADS / 32) * KMAX];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    uint32_t srcs[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) srcs[j] = a.src[lane * CPL + j];
    double dsum[CPL], nsum[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) dsum[j] = nsum[j] = 0.0;

    for (uint32_t k = gw; k < a.nseg; k += nw) {
        const uint4 sg = a.seg[k]; /* row, eb, ee, slot */
        float acc[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) acc[j] = 0.0f;
        for (uint32_t e0 = sg.y; e0 < sg.z; e0 += 32u) {
            const uint32_t n = min(32u, sg.z - e0);
            const uint32_t mine = lane < n ? __ldg(a.col + e0 + lane) : 0u;
            uint32_t j = 0;
            for (; j + 4 <= n; j += 4) { /* four row gathers in flight */
                float x0[CPL], x1[CPL], x2[CPL], x3[CPL];
                const uint32_t u0 = __shfl_sync(FULL, mine, j), u1 = __shfl_sync(FULL, mine, j + 1);
                const uint32_t u2 = __shfl_sync(FULL, mine, j + 2), u3 = __shfl_sync(FULL, mine, j + 3);
                load_row<CPL>(a.c_old + (size_t)u0 * a.kp + lane * CPL, x0);
                load_row<CPL>(a.c_old + (size_t)u1 * a.kp + lane * CPL, x1);
                load_row<CPL>(a.c_old + (size_t)u2 * a.kp + lane * CPL, x2);
                load_row<CPL>(a.c_old + (size_t)u3 * a.kp + lane * CPL, x3);
#pragma unroll
                for (int c = 0; c < CPL; ++c) acc[c] = (((acc[c] + x0[c]) + x1[c]) + x2[c]) + x3[c];
            }
            for (; j < n; ++j) {
                float x0[CPL];
                const uint32_t u0 = __shfl_sync(FULL, mine, j);
                load_row<CPL>(a.c_old + (size_t)u0 * a.kp + lane * CPL, x0);
#pragma unroll
                for (int c = 0; c < CPL; ++c) acc[c] += x0[c];
            }
        }
        if (sg.w == NONE) ppr_apply<CPL>(a, sg.x, acc, srcs, lane, dsum, nsum);
        else store_row<CPL>(a.partial + (size_t)sg.w * a.kp + lane * CPL, acc);
    }
    block_columns<CPL>(a, dsum, nsum, s_part, blockIdx.x);
}

/* rows of more than one segment (partials in segment order), the constant
 * vertices in sweeps 0 and 1, then — in the last block — the fixed-order
 * per-column residual reduction and the stopping test */
template <int CPL>
__global__ void __launch_bounds__(PPR_THREADS) k_ppr_fix(PprArgs a, int sweep, int const_pass) {
    if (*(volatile const int *)a.done) return;
    __shared__ double2 s_part[(PPR_THREADS / 32) * KMAX];
    __shared__ double s_res[KMAX];
    __shared__ int s_last;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    uint32_t srcs[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) srcs[j] = a.src[lane * CPL + j];
    double dsum[CPL], nsum[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) dsum[j] = nsum[j] = 0.0;
    for (uint32_t k = gw; k < a.nmulti; k += nw) {
        const uint4 m = a.multi[k]; /* row, first slot, count */
        float acc[CPL], x[CPL];
        load_row<CPL>(a.partial + (size_t)m.y * a.kp + lane * CPL, acc);
        for (uint32_t s = 1; s < m.z; ++s) {
            load_row<CPL>(a.partial + (size_t)(m.y + s) * a.kp + lane * CPL, x);
#pragma unroll
            for (int c = 0; c < CPL; ++c) acc[c] += x[c];
        }
        ppr_apply<CPL>(a, m.x, acc, srcs, lane, dsum, nsum);
    }
    if (const_pass) {
        float zero[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) zero[c] = 0.0f;
        for (uint32_t i = gw; i < a.nzero; i += nw) ppr_apply<CPL>(a, a.zero_rows[i], zero, srcs, lane, dsum, nsum);
    }
    block_columns<CPL>(a, dsum, nsum, s_part, a.nbseg + blockIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const uint32_t nb = a.nbseg + gridDim.x;
    for (uint32_t c = threadIdx.x; c < KMAX; c += blockDim.x) {
        double x = 0.0, y = 0.0;
        if (c < a.k) {
            for (uint32_t b = 0; b < nb; ++b) {
                const double2 p = __ldcg(a.bpart + (size_t)b * a.kp + c);
                x += p.x;
                y += p.y;
            }
            if (!const_pass) y += a.norm_const[c];
        }
        s_res[c] = (c < a.k && y > 0.0) ? x / y : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double worst = 0.0;
        for (uint32_t c = 0; c < a.k; ++c) worst = s_res[c] > worst ? s_res[c] : worst;
        a.res_log[sweep] = worst;
        *a.last_res = worst;
        *a.sweeps_done = sweep + 1;
        if (a.tol > 0.0 && worst <= a.tol) *a.done = 1;
        *a.ticket = 0u;
    }
}

__global__ void k_ppr_seed(const uint32_t *__restrict__ src, uint32_t k, uint32_t kp, const uint32_t *__restrict__ outdeg,
                           float *__restrict__ r, float *__restrict__ c) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const uint32_t v = src[j], od = outdeg[v];
    r[(size_t)v * kp + j] = 1.0f;
    c[(size_t)v * kp + j] = od ? __fdiv_rn(1.0f, (float)od) : 0.0f;
}

}  // namespace

/* Segments of the in-CSR for the batched sweeps, built once per graph. */
struct PprPlan {
    uint32_t nseg = 0, nmulti = 0, nzero = 0, nslots = 0;
    dbuf<uint4> seg, multi;
    dbuf<uint32_t> zero_rows;
    std::vector<uint32_t> indeg; /* host copy: constant-vertex test of the sources */
};

void free_ppr_plan(PprPlan *p) { delete p; }

static int ensure_ppr_plan(gcg_graph *g) {
    if (g->pplan) return GCG_OK;
    const uint32_t nv = g->nv;
    std::vector<uint32_t> rp((size_t)nv + 1);
    GCG_CUDA(cudaMemcpy(rp.data(), g->in_rowptr.get(), ((size_t)nv + 1) * 4, cudaMemcpyDeviceToHost));
    std::vector<uint4> seg, multi;
    std::vector<uint32_t> zero;
    PprPlan *p = new PprPlan();
    p->indeg.resize(nv);
    uint32_t slot = 0;
    for (uint32_t v = 0; v < nv; ++v) {
        const uint32_t b = rp[v], e = rp[v + 1], d = e - b;
        p->indeg[v] = d;
        if (d == 0) {
            zero.push_back(v);
            continue;
        }
        const uint32_t ns = (d + SEG - 1) / SEG;
        if (ns == 1) {
            seg.push_back(make_uint4(v, b, e, NONE));
        } else {
            multi.push_back(make_uint4(v, slot, ns, 0u));
            for (uint32_t s = 0; s < ns; ++s)
                seg.push_back(make_uint4(v, b + s * SEG, std::min(e, b + (s + 1) * SEG), slot + s));
            slot += ns;
        }
    }
    p->nseg = (uint32_t)seg.size();
    p->nmulti = (uint32_t)multi.size();
    p->nzero = (uint32_t)zero.size();
    p->nslots = slot;
    if (p->seg.alloc(std::max<size_t>(seg.size(), 1)) || p->multi.alloc(std::max<size_t>(multi.size(), 1)) ||
        p->zero_rows.alloc(std::max<size_t>(zero.size(), 1))) {
        delete p;
        return GCG_ERR_NOMEM;
    }
    cudaMemcpy(p->seg.get(), seg.data(), seg.size() * sizeof(uint4), cudaMemcpyHostToDevice);
    cudaMemcpy(p->multi.get(), multi.data(), multi.size() * sizeof(uint4), cudaMemcpyHostToDevice);
    cudaMemcpy(p->zero_rows.get(), zero.data(), zero.size() * 4, cudaMemcpyHostToDevice);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        delete p;
        return fail(GCG_ERR_CUDA, std::string("ppr plan: ") + cudaGetErrorString(e));
    }
    g->pplan = p;
    return GCG_OK;
}

namespace {

struct PprGroup {
    dbuf<float> r, c, partial;
    dbuf<double2> bpart;
    dbuf<uint32_t> src, ctl;
    dbuf<double> dres, norm_const;
};

template <int CPL>
int ppr_group(gcg_graph *g, const PprPlan &pl, const uint32_t *src_host, uint32_t k, const gcg_pr_params *p,
              float *out, uint32_t out_pitch, gcg_pr_stats *st, std::vector<double> *res_log) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv, kp = 32u * CPL;
    const int max_sweeps = p->max_sweeps;
    const int nbseg = num_sms() * 4, nbfix = num_sms() * 2;
    PprGroup w;
    GCG_TRY(w.r.alloc((size_t)2 * nv * kp));
    GCG_TRY(w.c.alloc((size_t)2 * nv * kp));
    GCG_TRY(w.partial.alloc((size_t)std::max<uint32_t>(pl.nslots, 1) * kp));
    GCG_TRY(w.bpart.alloc((size_t)(nbseg + nbfix) * kp));
    GCG_TRY(w.src.alloc(kp));
    GCG_TRY(w.ctl.alloc(4));
    GCG_TRY(w.dres.alloc((size_t)max_sweeps + 1));
    GCG_TRY(w.norm_const.alloc(kp));
    std::vector<uint32_t> srcv(kp, NONE);
    std::vector<double> nc(kp, 0.0);
    for (uint32_t j = 0; j < k; ++j) {
        srcv[j] = src_host[j];
        if (pl.indeg[src_host[j]] == 0) nc[j] = fabs((double)(float)p->teleport);
    }
    GCG_CUDA(cudaMemcpyAsync(w.src.get(), srcv.data(), kp * 4, cudaMemcpyHostToDevice, s));
    GCG_CUDA(cudaMemcpyAsync(w.norm_const.get(), nc.data(), kp * 8, cudaMemcpyHostToDevice, s));
    GCG_CUDA(cudaMemsetAsync(w.ctl.get(), 0, 16, s));
    GCG_CUDA(cudaMemsetAsync(w.r.get(), 0, (size_t)nv * kp * 4, s));
    GCG_CUDA(cudaMemsetAsync(w.c.get(), 0, (size_t)nv * kp * 4, s));
    k_ppr_seed<<<(k + 255) / 256, 256, 0, s>>>(w.src.get(), k, kp, g->outdeg.get(), w.r.get(), w.c.get());
    GCG_LAUNCH_CHECK();

    PprArgs a;
    a.col = g->in_col.get();
    a.outdeg = g->outdeg.get();
    a.seg = pl.seg.get();
    a.multi = pl.multi.get();
    a.zero_rows = pl.zero_rows.get();
    a.nseg = pl.nseg;
    a.nmulti = pl.nmulti;
    a.nzero = pl.nzero;
    a.kp = kp;
    a.k = k;
    a.src = w.src.get();
    a.partial = w.partial.get();
    a.bpart = w.bpart.get();
    a.nbseg = (uint32_t)nbseg;
    a.ticket = w.ctl.get();
    a.done = (int *)(w.ctl.get() + 1);
    a.sweeps_done = (int *)(w.ctl.get() + 2);
    a.res_log = w.dres.get();
    a.last_res = w.dres.get() + max_sweeps;
    a.norm_const = w.norm_const.get();
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.tol = p->tol;

    const bool time_sweeps = (p->flags & GCG_PR_TIME_SWEEPS) != 0;
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    std::vector<cudaEvent_t> sev;
    GCG_CUDA(cudaEventRecord(ev0, s));
    int launched = 0, done = 0;
    const size_t mat = (size_t)nv * kp;
    while (launched < max_sweeps && !done) {
        const int n = std::min(4, max_sweeps - launched);
        for (int i = 0; i < n; ++i) {
            const int sw = launched + i;
            a.r_old = w.r.get() + (size_t)(sw & 1) * mat;
            a.c_old = w.c.get() + (size_t)(sw & 1) * mat;
            a.r_new = w.r.get() + (size_t)((sw + 1) & 1) * mat;
            a.c_new = w.c.get() + (size_t)((sw + 1) & 1) * mat;
            if (time_sweeps) {
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, s);
                k_ppr_seg<CPL><<<nbseg, PPR_THREADS, 0, s>>>(a);
                cudaEventRecord(e1, s);
                sev.push_back(e0);
                sev.push_back(e1);
            } else {
                k_ppr_seg<CPL><<<nbseg, PPR_THREADS, 0, s>>>(a);
            }
            k_ppr_fix<CPL><<<nbfix, PPR_THREADS, 0, s>>>(a, sw, sw < 2 ? 1 : 0);
        }
        GCG_LAUNCH_CHECK();
        launched += n;
        if (p->tol > 0.0) {
            int h = 0;
            GCG_CUDA(cudaMemcpyAsync(&h, a.done, sizeof(int), cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            done = h;
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    uint32_t ctl[4];
    GCG_CUDA(cudaMemcpy(ctl, w.ctl.get(), sizeof(ctl), cudaMemcpyDeviceToHost));
    const int sweeps = (int)ctl[2];
    double seg_ms = 0.0;
    int timed = 0;
    for (size_t i = 0; i + 1 < sev.size(); i += 2) {
        if ((int)(i / 2) < sweeps) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, sev[i], sev[i + 1]);
            seg_ms += t;
            ++timed;
        }
        cudaEventDestroy(sev[i]);
        cudaEventDestroy(sev[i + 1]);
    }
    double last = 0.0;
    GCG_CUDA(cudaMemcpy(&last, a.last_res, 8, cudaMemcpyDeviceToHost));
    if (res_log && sweeps > 0) {
        std::vector<double> lg((size_t)sweeps);
        GCG_CUDA(cudaMemcpy(lg.data(), w.dres.get(), (size_t)sweeps * 8, cudaMemcpyDeviceToHost));
        if (res_log->size() < lg.size()) res_log->resize(lg.size(), 0.0);
        for (size_t i = 0; i < lg.size(); ++i) (*res_log)[i] = std::max((*res_log)[i], lg[i]);
    }
    const float *res = w.r.get() + (size_t)(sweeps & 1) * mat;
    GCG_CUDA(cudaMemcpy2DAsync(out, (size_t)out_pitch * 4, res, (size_t)kp * 4, (size_t)k * 4, nv, cudaMemcpyDefault,
                               s));
    GCG_CUDA(cudaStreamSynchronize(s));
    st->sweeps = std::max(st->sweeps, sweeps);
    st->converged = st->converged && (int)ctl[1];
    st->residual = std::max(st->residual, last);
    st->device_ms += ms;
    st->sweep_kernel_ms += seg_ms;
    st->timed_sweeps += timed;
    st->kernel_launches += 1 + 2 * launched;
    return GCG_OK;
}

}  // namespace
}  // namespace gcg

using namespace gcg;

extern "C" int gcg_ppr_batched(gcg_graph *g, const uint32_t *sources, uint32_t nsources, const gcg_pr_params *params,
                               float *out, gcg_pr_stats *stats) {
    if (!g || !sources || !params || !out) return fail(GCG_ERR_INVALID, "gcg_ppr_batched: null argument");
    if (nsources == 0) return fail(GCG_ERR_INVALID, "gcg_ppr_batched: nsources must be > 0");
    if (params->mode != GCG_PR_JACOBI || params->init_rank || params->source != GCG_NO_SOURCE)
        return fail(GCG_ERR_UNSUPPORTED,
                    "gcg_ppr_batched: Jacobi from the source indicators only (no init_rank, no source field)");
    if (params->max_sweeps < 0) return fail(GCG_ERR_INVALID, "gcg_ppr_batched: max_sweeps < 0");
    std::vector<uint32_t> src(nsources);
    GCG_CUDA(cudaMemcpy(src.data(), sources, (size_t)nsources * 4, cudaMemcpyDefault));
    for (uint32_t j = 0; j < nsources; ++j)
        if (src[j] >= g->nv) return fail(GCG_ERR_INVALID, "gcg_ppr_batched: source id >= num_vertices");
    GCG_TRY(ensure_ppr_plan(g));
    gcg_pr_stats st = {0, 1, 0.0, 0.0, 0.0, 0, 0};
    std::vector<double> lg;
    for (uint32_t g0 = 0; g0 < nsources; g0 += KMAX) {
        const uint32_t k = std::min(KMAX, nsources - g0);
        int rc;
        if (k <= 32) rc = ppr_group<1>(g, *g->pplan, src.data() + g0, k, params, out + g0, nsources, &st, &lg);
        else if (k <= 64) rc = ppr_group<2>(g, *g->pplan, src.data() + g0, k, params, out + g0, nsources, &st, &lg);
        else if (k <= 128) rc = ppr_group<4>(g, *g->pplan, src.data() + g0, k, params, out + g0, nsources, &st, &lg);
        else rc = ppr_group<8>(g, *g->pplan, src.data() + g0, k, params, out + g0, nsources, &st, &lg);
        if (rc != GCG_OK) return rc;
    }
    if (params->residuals && !lg.empty()) GCG_TRY(copy_out(params->residuals, lg.data(), lg.size() * 8, g->stream));
    if (stats) *stats = st;
    return GCG_OK;
}
