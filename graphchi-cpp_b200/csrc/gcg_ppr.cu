/*
 * Batched personalised PageRank: k sources at once as a dense rank matrix.
 *
 * No reference counterpart (the reference runs one vector per engine run,
 * example_apps/pagerank.cpp); the per-source semantics are those of the
 * personalised scalar path: r_s[v] = (float)(tele_s(v) + damping*(double)sum_{u->v}
 * c_s[u]) with tele_s(v) = teleport if v == source_s else 0, c_s[u] = r_s[u]/outdeg[u]
 * in float, r_s starting at the indicator of source_s, and each source stopping
 * after its own first sweep with normalised L1 change (FP64) <= tol.
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
 * residuals are reduced in a fixed order. A column that converges is copied to the
 * result at that sweep (k_ppr_retire) and keeps being swept in place; when the
 * columns still iterating fit a layout at most 3/4 as wide (widths 256, 192, 128,
 * 96, 64, 32), they are compacted into it.
 * Algorithmic traffic per sweep: E*(4 + 4*kp) + 3*V*4*kp bytes.
 */
#include <math.h>

#include <string.h>

#include <algorithm>
#include <memory>
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
    } else if constexpr (CPL == 6) {
        const float2 a = __ldg((const float2 *)p), b = __ldg((const float2 *)p + 1), c = __ldg((const float2 *)p + 2);
        x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y; x[4] = c.x; x[5] = c.y;
    } else if constexpr (CPL == 4) {
        const float4 a = __ldg((const float4 *)p);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    } else if constexpr (CPL == 3) {
        x[0] = __ldg(p); x[1] = __ldg(p + 1); x[2] = __ldg(p + 2);
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
    } else if constexpr (CPL == 6) {
        ((float2 *)p)[0] = make_float2(x[0], x[1]);
        ((float2 *)p)[1] = make_float2(x[2], x[3]);
        ((float2 *)p)[2] = make_float2(x[4], x[5]);
    } else if constexpr (CPL == 4) {
        ((float4 *)p)[0] = make_float4(x[0], x[1], x[2], x[3]);
    } else if constexpr (CPL == 3) {
        p[0] = x[0]; p[1] = x[1]; p[2] = x[2];
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
    int *col_sweeps;          /* per column: 0 while iterating, else the sweeps after which it converged */
    double *col_res;          /* per column: residual of its last iterated sweep */
    double teleport, damping, tol;
};

/* apply one row: r' = tele + damping*sum, c' = r'/outdeg, residual per column */
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
        for (uint32_t i = gw; i < a.nzero; i += nw)
            ppr_apply<CPL>(a, a.zero_rows[i], zero, srcs, lane, dsum, nsum);
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
    __shared__ int s_act[KMAX];
    /* per column: residual of this sweep; a column stops after its own first
     * sweep with residual <= tol (it keeps being swept in place until the next
     * compaction, but its answer is taken at that sweep) */
    for (uint32_t c = threadIdx.x; c < KMAX; c += blockDim.x) {
        double x = 0.0, y = 0.0;
        int act = 0;
        s_res[c] = 0.0;
        if (c < a.k && a.col_sweeps[c] == 0) {
            for (uint32_t b = 0; b < nb; ++b) {
                const double2 p = __ldcg(a.bpart + (size_t)b * a.kp + c);
                x += p.x;
                y += p.y;
            }
            if (!const_pass) y += a.norm_const[c];
            const double res = y > 0.0 ? x / y : 0.0;
            s_res[c] = res;
            a.col_res[c] = res;
            if (a.tol > 0.0 && res <= a.tol) a.col_sweeps[c] = sweep + 1;
            else act = 1;
        }
        s_act[c] = act;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double worst = 0.0;
        int active = 0;
        for (uint32_t c = 0; c < a.k; ++c) {
            worst = s_res[c] > worst ? s_res[c] : worst;
            active += s_act[c];
        }
        a.res_log[sweep] = worst;
        *a.last_res = worst;
        *a.sweeps_done = sweep + 1;
        if (active == 0) *a.done = 1;
        *a.ticket = 0u;
    }
}

/* the columns that converged in this sweep (col_sweeps == sweep + 1) are copied
 * from the sweep's rank matrix to their place in the result */
__global__ void __launch_bounds__(256) k_ppr_retire(const float *__restrict__ r, uint32_t kp, uint32_t k, uint32_t nv,
                                                    const int *__restrict__ col_sweeps, int sweep_done,
                                                    const uint32_t *__restrict__ gcol, float *__restrict__ dst,
                                                    size_t dpitch) {
    __shared__ uint32_t s_l[KMAX], s_g[KMAX];
    __shared__ uint32_t s_n;
    if (threadIdx.x == 0) {
        uint32_t n = 0;
        for (uint32_t c = 0; c < k; ++c)
            if (col_sweeps[c] == sweep_done) {
                s_l[n] = c;
                s_g[n] = gcol[c];
                ++n;
            }
        s_n = n;
    }
    __syncthreads();
    const uint32_t n = s_n;
    if (n == 0) return;
    const uint64_t tot = (uint64_t)nv * n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < tot; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / n), j = (uint32_t)(i % n);
        dst[(size_t)v * dpitch + s_g[j]] = r[(size_t)v * kp + s_l[j]];
    }
}

/* copies columns of a V x kp matrix: dst[v*dpitch + dcol[j]] = src[v*kp + scol[j]] */
__global__ void k_ppr_columns(const float *__restrict__ src, uint32_t kp, uint32_t nv, const uint32_t *__restrict__ scol,
                              const uint32_t *__restrict__ dcol, uint32_t n, float *__restrict__ dst, size_t dpitch) {
    const uint64_t tot = (uint64_t)nv * n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < tot; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / n), j = (uint32_t)(i % n);
        dst[(size_t)v * dpitch + dcol[j]] = src[(size_t)v * kp + scol[j]];
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

/* rank / contribution matrices of one layout width, and its per-column state */
struct PprLayout {
    uint32_t cpl = 0, kp = 0, k = 0;  /* columns per lane, padded width, columns in use */
    dbuf<float> r, c;                 /* 2 x V x kp each (the two sweep parities) */
    dbuf<uint32_t> src, gcol;         /* kp source ids (NONE for padding); group column of each */
    dbuf<double> norm_const, col_res; /* kp */
    dbuf<int> col_sweeps;             /* kp */
    int alloc(uint32_t nv, uint32_t cpl_) {
        cpl = cpl_;
        kp = 32u * cpl_;
        const size_t mat = (size_t)nv * kp;
        if (r.alloc(2 * mat) || c.alloc(2 * mat) || src.alloc(kp) || gcol.alloc(kp) || norm_const.alloc(kp) ||
            col_res.alloc(kp) || col_sweeps.alloc(kp))
            return GCG_ERR_NOMEM;
        return GCG_OK;
    }
};

/* lanes hold 1, 2, 3, 4, 6 or 8 columns: widths 32 .. 256 */
uint32_t cpl_for(uint32_t n) {
    return n <= 32 ? 1u : n <= 64 ? 2u : n <= 96 ? 3u : n <= 128 ? 4u : n <= 192 ? 6u : 8u;
}

template <int CPL>
void ppr_sweep(const PprArgs &a, int nbseg, int nbfix, int sw, cudaStream_t s, std::vector<cudaEvent_t> *sev) {
    if (sev) {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        k_ppr_seg<CPL><<<nbseg, PPR_THREADS, 0, s>>>(a);
        cudaEventRecord(e1, s);
        sev->push_back(e0);
        sev->push_back(e1);
    } else {
        k_ppr_seg<CPL><<<nbseg, PPR_THREADS, 0, s>>>(a);
    }
    k_ppr_fix<CPL><<<nbfix, PPR_THREADS, 0, s>>>(a, sw, sw < 2 ? 1 : 0);
}

void ppr_sweep_any(uint32_t cpl, const PprArgs &a, int nbseg, int nbfix, int sw, cudaStream_t s,
                   std::vector<cudaEvent_t> *sev) {
    switch (cpl) {
        case 1: ppr_sweep<1>(a, nbseg, nbfix, sw, s, sev); break;
        case 2: ppr_sweep<2>(a, nbseg, nbfix, sw, s, sev); break;
        case 3: ppr_sweep<3>(a, nbseg, nbfix, sw, s, sev); break;
        case 4: ppr_sweep<4>(a, nbseg, nbfix, sw, s, sev); break;
        case 6: ppr_sweep<6>(a, nbseg, nbfix, sw, s, sev); break;
        default: ppr_sweep<8>(a, nbseg, nbfix, sw, s, sev); break;
    }
}

/* columns scol[j] of src (V x kp) -> columns dcol[j] of dst (row pitch dpitch) */
int copy_columns(const float *src, uint32_t kp, uint32_t nv, const std::vector<uint32_t> &scol,
                 const std::vector<uint32_t> &dcol, float *dst, size_t dpitch, cudaStream_t s) {
    const uint32_t n = (uint32_t)scol.size();
    if (n == 0 || nv == 0) return GCG_OK;
    tbuf<uint32_t> d;
    GCG_TRY(d.alloc(2 * (size_t)n, s));
    std::vector<uint32_t> h(scol);
    h.insert(h.end(), dcol.begin(), dcol.end());
    GCG_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * 4, cudaMemcpyHostToDevice, s));
    const uint64_t tot = (uint64_t)nv * n;
    const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((tot + 255) / 256, num_sms() * 16ull));
    k_ppr_columns<<<blocks, 256, 0, s>>>(src, kp, nv, d.get(), d.get() + n, n, dst, dpitch);
    GCG_LAUNCH_CHECK();
    GCG_CUDA(cudaStreamSynchronize(s)); /* h is host stack memory */
    return GCG_OK;
}

/* One group of k <= 256 sources. Each column stops after its own first sweep
 * with residual <= tol (the scalar path's rule): it is copied to the result at
 * that sweep; whenever the columns still iterating fit a layout at most 3/4 as
 * wide, they are compacted into it, so later sweeps gather narrower rows. */
int ppr_group(gcg_graph *g, const PprPlan &pl, const uint32_t *src_host, uint32_t k, const gcg_pr_params *p,
              float *out, uint32_t out_pitch, gcg_pr_stats *st, std::vector<double> *res_log,
              std::vector<int> *col_sweeps) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    const int max_sweeps = p->max_sweeps;
    const int nbseg = num_sms() * 4, nbfix = num_sms() * 2;
    dbuf<float> partial, stage;
    dbuf<double2> bpart;
    dbuf<uint32_t> ctl;
    dbuf<double> dres;
    GCG_TRY(partial.alloc((size_t)std::max<uint32_t>(pl.nslots, 1) * KMAX));
    GCG_TRY(bpart.alloc((size_t)(nbseg + nbfix) * KMAX));
    GCG_TRY(ctl.alloc(4));
    GCG_TRY(dres.alloc((size_t)max_sweeps + 1));
    /* finished columns go straight to a device output, else to a staging matrix */
    const bool dev_out = is_device_ptr(out);
    float *res_dst = out;
    size_t res_pitch = out_pitch;
    if (!dev_out) {
        GCG_TRY(stage.alloc((size_t)nv * k));
        res_dst = stage.get();
        res_pitch = k;
    }
    std::vector<uint32_t> act(k); /* layout column -> group column */
    for (uint32_t j = 0; j < k; ++j) act[j] = j;
    std::vector<int> fin_sweeps(k, 0);
    std::vector<double> fin_res(k, 0.0);

    auto lay = std::make_unique<PprLayout>();
    GCG_TRY(lay->alloc(nv, cpl_for(k)));
    lay->k = k;
    auto upload_state = [&](PprLayout &L) -> int {
        std::vector<uint32_t> srcv(L.kp, NONE), gc(L.kp, 0u);
        std::vector<double> nc(L.kp, 0.0);
        for (uint32_t j = 0; j < L.k; ++j) {
            srcv[j] = src_host[act[j]];
            gc[j] = act[j];
            if (pl.indeg[srcv[j]] == 0) nc[j] = fabs((double)(float)p->teleport);
        }
        GCG_CUDA(cudaMemcpyAsync(L.src.get(), srcv.data(), L.kp * 4, cudaMemcpyHostToDevice, s));
        GCG_CUDA(cudaMemcpyAsync(L.gcol.get(), gc.data(), L.kp * 4, cudaMemcpyHostToDevice, s));
        GCG_CUDA(cudaMemcpyAsync(L.norm_const.get(), nc.data(), L.kp * 8, cudaMemcpyHostToDevice, s));
        GCG_CUDA(cudaMemsetAsync(L.col_sweeps.get(), 0, L.kp * 4, s));
        GCG_CUDA(cudaMemsetAsync(L.col_res.get(), 0, L.kp * 8, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        return GCG_OK;
    };
    GCG_TRY(upload_state(*lay));
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
    GCG_CUDA(cudaMemsetAsync(lay->r.get(), 0, (size_t)nv * lay->kp * 4, s));
    GCG_CUDA(cudaMemsetAsync(lay->c.get(), 0, (size_t)nv * lay->kp * 4, s));
    k_ppr_seed<<<(k + 255) / 256, 256, 0, s>>>(lay->src.get(), k, lay->kp, g->outdeg.get(), lay->r.get(), lay->c.get());
    GCG_LAUNCH_CHECK();

    PprArgs a;
    memset(&a, 0, sizeof(a));
    a.col = g->in_col.get();
    a.outdeg = g->outdeg.get();
    a.seg = pl.seg.get();
    a.multi = pl.multi.get();
    a.zero_rows = pl.zero_rows.get();
    a.nseg = pl.nseg;
    a.nmulti = pl.nmulti;
    a.nzero = pl.nzero;
    a.partial = partial.get();
    a.bpart = bpart.get();
    a.nbseg = (uint32_t)nbseg;
    a.ticket = ctl.get();
    a.done = (int *)(ctl.get() + 1);
    a.sweeps_done = (int *)(ctl.get() + 2);
    a.res_log = dres.get();
    a.last_res = dres.get() + max_sweeps;
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.tol = p->tol;
    auto bind = [&](PprLayout &L) {
        a.kp = L.kp;
        a.k = L.k;
        a.src = L.src.get();
        a.norm_const = L.norm_const.get();
        a.col_sweeps = L.col_sweeps.get();
        a.col_res = L.col_res.get();
    };
    bind(*lay);

    const bool time_sweeps = (p->flags & GCG_PR_TIME_SWEEPS) != 0;
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    std::vector<cudaEvent_t> sev;
    GCG_CUDA(cudaEventRecord(ev0, s));
    int sweep = 0, launches = 1, compactions = 0;
    bool done = false;
    std::vector<int> hsw(KMAX);
    std::vector<double> hres(KMAX);
    while (sweep < max_sweeps && !done) {
        const int n = std::min(4, max_sweeps - sweep);
        const size_t mat = (size_t)nv * lay->kp;
        for (int i = 0; i < n; ++i) {
            const int sw = sweep + i;
            a.r_old = lay->r.get() + (size_t)(sw & 1) * mat;
            a.c_old = lay->c.get() + (size_t)(sw & 1) * mat;
            a.r_new = lay->r.get() + (size_t)((sw + 1) & 1) * mat;
            a.c_new = lay->c.get() + (size_t)((sw + 1) & 1) * mat;
            ppr_sweep_any(lay->cpl, a, nbseg, nbfix, sw, s, time_sweeps ? &sev : nullptr);
            if (p->tol > 0.0)
                k_ppr_retire<<<num_sms(), 256, 0, s>>>(a.r_new, lay->kp, lay->k, nv, lay->col_sweeps.get(), sw + 1,
                                                       lay->gcol.get(), res_dst, res_pitch);
        }
        GCG_LAUNCH_CHECK();
        launches += (p->tol > 0.0 ? 3 : 2) * n;
        sweep += n;
        if (!(p->tol > 0.0)) continue;
        uint32_t h[4];
        GCG_CUDA(cudaMemcpyAsync(h, ctl.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaMemcpyAsync(hsw.data(), lay->col_sweeps.get(), lay->k * 4, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        if (h[1]) {
            done = true;
            sweep = (int)h[2];
            break;
        }
        uint32_t nact = 0;
        for (uint32_t j = 0; j < lay->k; ++j) nact += hsw[j] == 0;
        if (sweep >= max_sweeps || 4 * 32 * cpl_for(nact) > 3 * lay->kp) continue;
        /* compact the columns still iterating into a narrower layout (the others
         * are already in the result) */
        GCG_CUDA(cudaMemcpyAsync(hres.data(), lay->col_res.get(), lay->k * 8, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        const float *rcur = lay->r.get() + (size_t)(sweep & 1) * mat;
        const float *ccur = lay->c.get() + (size_t)(sweep & 1) * mat;
        std::vector<uint32_t> ks, kd, nact_cols;
        for (uint32_t j = 0; j < lay->k; ++j) {
            if (hsw[j]) {
                fin_sweeps[act[j]] = hsw[j];
                fin_res[act[j]] = hres[j];
            } else {
                ks.push_back(j);
                kd.push_back((uint32_t)nact_cols.size());
                nact_cols.push_back(act[j]);
            }
        }
        auto nxt = std::make_unique<PprLayout>();
        GCG_TRY(nxt->alloc(nv, cpl_for(nact)));
        nxt->k = nact;
        const size_t nmat = (size_t)nv * nxt->kp;
        GCG_CUDA(cudaMemsetAsync(nxt->r.get(), 0, 2 * nmat * 4, s));
        GCG_CUDA(cudaMemsetAsync(nxt->c.get(), 0, 2 * nmat * 4, s));
        for (int par = 0; par < 2; ++par) { /* both parities: rows not swept any more keep their values */
            GCG_TRY(copy_columns(rcur, lay->kp, nv, ks, kd, nxt->r.get() + (size_t)par * nmat, nxt->kp, s));
            GCG_TRY(copy_columns(ccur, lay->kp, nv, ks, kd, nxt->c.get() + (size_t)par * nmat, nxt->kp, s));
        }
        act = nact_cols;
        GCG_TRY(upload_state(*nxt));
        lay = std::move(nxt);
        bind(*lay);
        launches += 4;
        ++compactions;
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    uint32_t ctlh[4];
    GCG_CUDA(cudaMemcpy(ctlh, ctl.get(), sizeof(ctlh), cudaMemcpyDeviceToHost));
    const int sweeps = (int)ctlh[2];
    double seg_ms = 0.0;
    int timed = 0;
    for (size_t i = 0; i + 1 < sev.size(); i += 2) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, sev[i], sev[i + 1]) == cudaSuccess && (int)(i / 2) < sweeps) {
            seg_ms += t;
            ++timed;
        }
        cudaEventDestroy(sev[i]);
        cudaEventDestroy(sev[i + 1]);
    }
    cudaGetLastError();
    /* the columns still in the layout: final values are in the buffer of the last sweep */
    GCG_CUDA(cudaMemcpy(hsw.data(), lay->col_sweeps.get(), lay->k * 4, cudaMemcpyDeviceToHost));
    GCG_CUDA(cudaMemcpy(hres.data(), lay->col_res.get(), lay->k * 8, cudaMemcpyDeviceToHost));
    {
        /* columns that never converged: the buffer of the last sweep */
        std::vector<uint32_t> ks, kd;
        for (uint32_t j = 0; j < lay->k; ++j) {
            fin_sweeps[act[j]] = hsw[j] ? hsw[j] : sweeps;
            fin_res[act[j]] = hres[j];
            if (!hsw[j]) {
                ks.push_back(j);
                kd.push_back(act[j]);
            }
        }
        const float *rfin = lay->r.get() + (size_t)(sweeps & 1) * (size_t)nv * lay->kp;
        GCG_TRY(copy_columns(rfin, lay->kp, nv, ks, kd, res_dst, res_pitch, s));
        launches += ks.empty() ? 0 : 1;
    }
    if (res_log && sweeps > 0) {
        std::vector<double> lg((size_t)sweeps);
        GCG_CUDA(cudaMemcpy(lg.data(), dres.get(), (size_t)sweeps * 8, cudaMemcpyDeviceToHost));
        if (res_log->size() < lg.size()) res_log->resize(lg.size(), 0.0);
        for (size_t i = 0; i < lg.size(); ++i) (*res_log)[i] = std::max((*res_log)[i], lg[i]);
    }
    if (!dev_out)
        GCG_CUDA(cudaMemcpy2DAsync(out, (size_t)out_pitch * 4, stage.get(), (size_t)k * 4, (size_t)k * 4, nv,
                                   cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    bool conv = p->tol > 0.0;
    double worst = 0.0;
    int mx = 0;
    for (uint32_t j = 0; j < k; ++j) {
        mx = std::max(mx, fin_sweeps[j]);
        worst = std::max(worst, fin_res[j]);
        if (!(p->tol > 0.0 && fin_res[j] <= p->tol)) conv = false;
    }
    if (col_sweeps) col_sweeps->insert(col_sweeps->end(), fin_sweeps.begin(), fin_sweeps.end());
    st->sweeps = std::max(st->sweeps, mx);
    st->converged = st->converged && conv;
    st->residual = std::max(st->residual, worst);
    st->device_ms += ms;
    st->sweep_kernel_ms += seg_ms;
    st->timed_sweeps += timed;
    st->kernel_launches += launches;
    (void)compactions;
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
    std::vector<int> col_sweeps; /* sweeps each source took */
    for (uint32_t g0 = 0; g0 < nsources; g0 += KMAX) {
        const uint32_t k = std::min(KMAX, nsources - g0);
        GCG_TRY(ppr_group(g, *g->pplan, src.data() + g0, k, params, out + g0, nsources, &st, &lg, &col_sweeps));
    }
    if (params->residuals && !lg.empty()) GCG_TRY(copy_out(params->residuals, lg.data(), lg.size() * 8, g->stream));
    if (params->work_log && params->max_sweeps > 0) {
        /* cumulative work of the sources still iterating: sweep i updates every
         * vertex and gathers every in-edge once per source with more than i sweeps */
        const int S = params->max_sweeps;
        std::vector<uint64_t> active((size_t)S + 1, 0);
        for (int c : col_sweeps) ++active[(size_t)std::min(c, S)];
        std::vector<uint64_t> wl(2 * (size_t)S);
        uint64_t left = col_sweeps.size(), upd = 0, gat = 0;
        for (int i = 0; i < S; ++i) {
            left -= active[(size_t)i]; /* sources that took exactly i sweeps are done */
            upd += left * (uint64_t)g->nv;
            gat += left * g->ne;
            wl[2 * (size_t)i] = upd;
            wl[2 * (size_t)i + 1] = gat;
        }
        GCG_TRY(copy_out(params->work_log, wl.data(), wl.size() * 8, g->stream));
    }
    if (stats) *stats = st;
    return GCG_OK;
}
