/*
 * Device pieces of the Jacobi PageRank sweep shared by the single-graph engine
 * (gcg_pagerank.cu) and the multi-graph persistent launch (gcg_multi.cu): the
 * sweep arguments, cache-policy loads, the chunk loader, the hub-cache gather and
 * the warp-level chunk reduction, and the apply formula.
 */
#ifndef GCG_PR_DEVICE_CUH
#define GCG_PR_DEVICE_CUH

#include "gcg_internal.cuh"

namespace gcg {

constexpr int CH = 256;  /* edges per warp chunk */
constexpr int EPL = 8;   /* edges per lane */

/* ---- cache-policy loads --------------------------------------------------- */
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint4 ld_stream_v4(const uint32_t *p, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float ld_keep_f32(const float *p, uint64_t pol) {
    float r;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(p), "l"(pol));
    return r;
}

/* ---- bulk copies into shared memory (TMA), completion on an mbarrier ------ */
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    /* the initialised barrier is visible to the copy engine before any copy names it */
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
/* the calling thread's arrival, announcing `bytes` of copies that complete on bar */
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
/* global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16 */
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
/* bound on the polls of a barrier wait (each try_wait may itself suspend the
 * thread for a while): far above any copy's completion time */
constexpr long long MBAR_SPIN = 1ll << 22;

/* ---- sweep kernels ------------------------------------------------------ */
struct SweepArgs {
    /* graph / plan */
    const uint32_t *col, *outdeg;
    const uint8_t *heads;
    const uint32_t *chunk_nz, *nz_rows, *zero_rows;
    const uint4 *split;
    const uint32_t *long_split; /* indices into split of the rows spanning more than LONG_SPAN chunks */
    uint32_t nlong;
    uint64_t ne;
    uint32_t nchunks, nnz, nzero, nsplit;
    uint32_t hub; /* contribs of relabelled sources [0, hub) are cached in shared memory */
    const uint32_t *nz_cidx, *zero_cidx; /* relabelled ids of the nz / zero rows */
    /* state (contribs indexed by relabelled id) */
    const float *c_old;
    float *c_new;
    const float *r_nz_old; /* ranks of the vertices with in-edges, compact (nz order) */
    float *r_nz_new;
    const uint32_t *od_nz; /* their out-degrees, compact */
    const float *r_init;   /* full initial vector (residual of the first sweep) */
    float *nzsum, *head_part, *tail_part;
    double2 *block_res;
    uint32_t *ticket;
    int *done, *sweeps_done;
    double *res_log, *last_res;
    double teleport, damping, tol, norm_const;
    uint32_t source; /* personalisation vertex, or GCG_NO_SOURCE */
    uint32_t run;    /* edge kernel: each warp takes runs of this many consecutive chunks (>= 1) */
    double *delta_log; /* optional: per sweep, sum |r' - r| (FP64) */
    unsigned long long tex_old; /* texture object over c_old (edge kernel's texture-path gathers) */
    int *err;                   /* edge kernel: set when the hub copy's wait ran out */
    /* source tiers (vertex kernel): a row's sum is the sum over tiers k of
     * tier_sum[k][tier_idx[k * nnz + i]] (entries equal to GCG_NO_SOURCE: no
     * in-edge of the row in that tier), tiers added in order; ntiers <= 1: nzsum */
    uint32_t ntiers;
    const uint32_t *tier_idx;
    const float *tier_sum[4];
};

/* Column layout of a chunk. Lane l owns the 8 consecutive edges 8l..8l+7 of a
 * 256-edge chunk, but they are stored split in two halves so that each of the
 * lane's two 128-bit loads is part of one contiguous 512-byte warp access (16
 * full sectors) instead of a 1 KiB access using half of each of 32 sectors:
 * edge 8l+j (j < 4) sits at slot 4l+j, edge 8l+4+j at slot 128+4l+j. The array
 * holds whole chunks (padding slots are 0). */
__host__ __device__ __forceinline__ uint64_t chunk_slot(uint64_t e) {
    const uint64_t l = (e >> 3) & 31u, j = e & 7u;
    return (e & ~(uint64_t)(CH - 1)) + (j < 4 ? 4u * l + j : 128u + 4u * l + (j - 4u));
}

/* columns (streamed), head flags and starting row index of one chunk; ne is
 * the end of the edge range being swept (positions at or beyond it are masked) */
template <typename A>
__device__ __forceinline__ void load_chunk(const A &a, uint32_t ch, uint32_t lane, uint64_t pol, uint32_t (&col)[EPL],
                                           uint32_t &flags, uint32_t &nvalid, uint32_t &base, uint64_t ne) {
    const uint64_t c0 = (uint64_t)ch * CH;
    const uint64_t e = c0 + (uint64_t)EPL * lane;
    nvalid = e < ne ? (uint32_t)((ne - e) < EPL ? (ne - e) : EPL) : 0u;
    const uint4 x = ld_stream_v4(a.col + c0 + 4u * lane, pol);
    const uint4 y = ld_stream_v4(a.col + c0 + 128u + 4u * lane, pol);
    col[0] = x.x; col[1] = x.y; col[2] = x.z; col[3] = x.w;
    col[4] = y.x; col[5] = y.y; col[6] = y.z; col[7] = y.w;
    if (nvalid < EPL) {
#pragma unroll
        for (int j = 0; j < EPL; ++j)
            if ((uint32_t)j >= nvalid) col[j] = 0u;
    }
    flags = nvalid ? ((uint32_t)a.heads[e >> 3] & ((1u << nvalid) - 1u)) : 0u;
    base = a.chunk_nz[ch];
}

/* L2-coherent load (no non-coherent texture path) for data that the same
 * kernel launch rewrote before a grid barrier */
__device__ __forceinline__ float ld_cg_keep_f32(const float *p, uint64_t pol) {
    float r;
    asm volatile("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(p), "l"(pol) : "memory");
    return r;
}

/* hub cache: contribs of the highest out-degree sources (relabelled 0..hub-1);
 * the caller synchronises the block afterwards */
template <typename A>
__device__ __forceinline__ void load_hub(const A &a, float *s_hub) {
    const uint32_t n4 = a.hub >> 2;
    const float4 *src4 = (const float4 *)a.c_old;
    float4 *dst4 = (float4 *)s_hub;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) dst4[i] = __ldcg(src4 + i);
    for (uint32_t i = (n4 << 2) + threadIdx.x; i < a.hub; i += blockDim.x) s_hub[i] = __ldcg(a.c_old + i);
}

/* contribs of a chunk's sources: hub sources from shared memory, the rest from
 * L2/HBM (kept in L2). COHERENT selects loads that see writes made earlier in
 * the same launch. */
template <bool COHERENT = false, typename A>
__device__ __forceinline__ void gather_chunk(const A &a, const uint32_t (&col)[EPL], uint32_t nvalid,
                                             const float *s_hub, uint64_t pol_keep, float (&val)[EPL]) {
#pragma unroll
    for (int j = 0; j < EPL; ++j) {
        const uint32_t x = col[j];
        float v = 0.0f;
        if ((uint32_t)j < nvalid) {
            if (x < a.hub) v = s_hub[x];
            else v = COHERENT ? ld_cg_keep_f32(a.c_old + x, pol_keep) : ld_keep_f32(a.c_old + x, pol_keep);
        }
        val[j] = v;
    }
}

/* Value types of the chunk reduction: float (PageRank sums) and Agg3 (three
 * channels: sum, max, sum). vadd is the reduction; for float it is the plain
 * IEEE sum, so the PageRank instantiation computes exactly a + b. */
struct Agg3 {
    float s, m, t;
};
__device__ __forceinline__ float vzero(float) { return 0.0f; }
__device__ __forceinline__ Agg3 vzero(Agg3) { return Agg3{0.0f, 0.0f, 0.0f}; }
__device__ __forceinline__ float vadd(float x, float y) { return x + y; }
__device__ __forceinline__ Agg3 vadd(Agg3 x, Agg3 y) { return Agg3{x.s + y.s, fmaxf(x.m, y.m), x.t + y.t}; }
__device__ __forceinline__ float vshfl_up(float x, int o) { return __shfl_up_sync(0xFFFFFFFFu, x, o); }
__device__ __forceinline__ Agg3 vshfl_up(Agg3 x, int o) {
    return Agg3{__shfl_up_sync(0xFFFFFFFFu, x.s, o), __shfl_up_sync(0xFFFFFFFFu, x.m, o),
                __shfl_up_sync(0xFFFFFFFFu, x.t, o)};
}

/* Warp reduction of one chunk into row values. Rows that start and end inside the
 * chunk are written to nzsum; a row that began in an earlier chunk leaves its
 * part in head_part[ch], a row that continues into the next chunk leaves its
 * part in tail_part[ch] (both completed in chunk order by the fix-up pass).
 * ne is the end of the edge range being swept. A supplies heads; R supplies
 * nzsum, head_part and tail_part of value type V. */
template <typename A, typename R, typename V>
__device__ __forceinline__ void reduce_chunk_to(const A &a, const R &o, uint32_t ch, uint32_t lane,
                                                const V (&val)[EPL], uint32_t flags, uint32_t nvalid, uint32_t base,
                                                uint64_t ne) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint64_t e0 = (uint64_t)ch * CH;
    const uint32_t head0 = __shfl_sync(FULL, flags, 0) & 1u;
    const uint32_t nh_lane = __popc(flags);
    uint32_t incl = nh_lane;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(FULL, incl, d);
        if (lane >= (uint32_t)d) incl += y;
    }
    const uint32_t H = incl - nh_lane; /* heads in earlier lanes of this chunk */
    const uint32_t Htot = __shfl_sync(FULL, incl, 31);
    const uint32_t rowbase = base + (head0 ? 0u : 1u) + H; /* row started by this lane's first head */

    /* in-lane segments: rows that start and end inside this lane are final */
    const V zero = vzero(val[0]);
    V run = zero, pre = zero;
    uint32_t nh = 0;
#pragma unroll
    for (int j = 0; j < EPL; ++j) {
        if ((uint32_t)j < nvalid) {
            if ((flags >> j) & 1u) {
                if (nh == 0) pre = run;
                else o.nzsum[rowbase + nh - 1] = run;
                ++nh;
                run = zero;
            }
            run = vadd(run, val[j]);
        }
    }
    /* warp segmented inclusive scan of (lane has a head, lane tail value) */
    int finc = nh > 0;
    V vinc = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int fu = __shfl_up_sync(FULL, finc, d);
        V vu = vshfl_up(vinc, d);
        if (lane >= (uint32_t)d) {
            if (!finc) vinc = vadd(vu, vinc);
            finc |= fu;
        }
    }
    const V prev = vshfl_up(vinc, 1);
    const V carry = lane ? prev : zero;
    if (nh > 0) {
        /* the row that ends at this lane's first head */
        const V sv = vadd(carry, pre);
        if (H == 0 && !head0) o.head_part[ch] = sv;                /* began in an earlier chunk */
        else if (!(lane == 0 && head0)) o.nzsum[rowbase - 1] = sv; /* began in an earlier lane */
    }
    /* the chunk's last row */
    const uint32_t L = (ne - e0 >= (uint64_t)CH) ? 31u : (uint32_t)((ne - 1 - e0) / EPL);
    if (lane == L) {
        if (Htot == 0) {
            o.head_part[ch] = vinc; /* the whole chunk lies inside one row */
        } else {
            const bool ends_here = (e0 + CH >= ne) || (a.heads[(e0 + CH) >> 3] & 1u);
            const uint32_t idx = base + (head0 ? 0u : 1u) + Htot - 1;
            if (ends_here) o.nzsum[idx] = vinc;
            else o.tail_part[ch] = vinc;
        }
    }
}

template <typename A>
__device__ __forceinline__ void reduce_chunk(const A &a, uint32_t ch, uint32_t lane, const float (&val)[EPL],
                                             uint32_t flags, uint32_t nvalid, uint32_t base, uint64_t ne) {
    reduce_chunk_to(a, a, ch, lane, val, flags, nvalid, base, ne);
}

constexpr int EDGE_THREADS = 1024;
constexpr uint32_t HUB_MAX = 49152; /* 192 KB of shared memory */
/* Default hub of the edge kernel: the largest that fits the 164 KB shared-memory
 * carve-out together with the kernel's 16 bytes of static shared memory (the
 * hub copy's mbarrier) and the 1 KB the driver reserves per block, leaving
 * ~92 KB of L1; one more byte moves the SM to the 196 KB carve-out and cuts L1
 * by a third (the edge kernel then takes 16 % longer at R-MAT scale 24). */
constexpr uint32_t HUB_DEFAULT = 41724;
constexpr uint32_t RUN_DEFAULT = 1; /* with texture gathers, 0.4 % faster than runs of 2 */

/* Sweep workspace of one graph, reused across calls. */
struct PrWork {
    dbuf<float> r, c, nzsum, parts, rnz;
    dbuf<double2> bres;
    dbuf<uint32_t> ctl;
    dbuf<double> dres;
    int *h_flags = nullptr; /* pinned: done flags copied back per chunk of sweeps */
    /* texture objects over the two contribution buffers (0: not available, the
     * edge kernel then gathers with plain loads) */
    unsigned long long tex[2] = {0, 0};
    ~PrWork() {
        if (h_flags) host_free(h_flags);
        for (unsigned long long t : tex)
            if (t) cudaDestroyTextureObject((cudaTextureObject_t)t);
    }
};

/* Rows that cross chunk boundaries: a row spanning at most LONG_SPAN chunks is
 * summed by one thread in chunk order (tail part, then the head parts). A longer
 * row is summed by one warp in one fixed order (the single-graph fix-up and the
 * batch kernel alike): LONG_GROUPS groups of 32 lanes; lane l of group g adds the head parts
 * of chunks cs+1+32g+l, cs+1+32g+l+256, ... in order; each group is reduced by
 * an xor tree over its 32 lanes; the group sums are added in group order, and
 * the tail part last. */
constexpr uint32_t LONG_SPAN = 8;
constexpr int LONG_GROUPS = 8;

template <bool COHERENT>
__device__ __forceinline__ float long_row_group(const float *head_part, uint32_t cs, uint32_t ce, int grp,
                                                uint32_t lane) {
    float s = 0.0f;
    for (uint32_t c = cs + 1 + 32u * (uint32_t)grp + lane; c <= ce; c += 32u * LONG_GROUPS)
        s += COHERENT ? __ldcg(head_part + c) : head_part[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    return s;
}

/* the whole long-row sum by one warp (every lane returns it) */
template <bool COHERENT>
__device__ __forceinline__ float long_row_sum_warp(const float *head_part, uint32_t cs, uint32_t ce,
                                                   uint32_t lane) {
    float t = 0.0f;
#pragma unroll 1
    for (int grp = 0; grp < LONG_GROUPS; ++grp) t += long_row_group<COHERENT>(head_part, cs, ce, grp, lane);
    return t;
}

/* Source tiers of the edge phase. The sources (relabelled by out-degree) are cut
 * into tiers of `width` ids: tier k >= 1 holds the edges whose source lies in
 * [k * width, (k + 1) * width), tier 0 every other edge (the hub [0, width) and
 * the sources past the last tier). Each tier is its own edge array grouped by
 * row (columns relative to the tier's first id) with its own chunk structure,
 * so its edge pass keeps the tier's contributions in shared memory: tier k >= 1
 * needs no global gathers at all. A row's sum is its tiers' partial sums added
 * in tier order. */
constexpr int MAX_TIERS = 4;
struct EdgeTier {
    uint64_t ne = 0;
    uint32_t nchunks = 0, nrows = 0, nsplit = 0, nlong = 0;
    uint32_t first = 0; /* relabelled id of column value 0 */
    uint32_t hub = 0;   /* contributions [first, first + hub) staged in shared memory */
    dbuf<uint32_t> col, head_bits, chunk_nz, long_split;
    dbuf<uint4> split;
    dbuf<float> nzsum, parts;
};
struct TierPlan {
    int ntiers = 0; /* built for this many tiers (0: not built) */
    uint32_t width = 0;
    EdgeTier t[MAX_TIERS];
    dbuf<uint32_t> idx; /* ntiers x nnz: each row's index in tier k's rows, or GCG_NO_SOURCE */
};

struct ChunkPlan {
    PrWork work;
    TierPlan tiers;
    uint32_t tune_tiers = 1; /* source tiers of the edge phase (1: one pass) */
    uint32_t nchunks = 0, nnz = 0, nzero = 0, nsplit = 0;
    /* rows are taken in relabelled order (row j is the vertex relabelled j), so
     * the vertex pass writes contributions in sequence; false only for a union
     * whose relabelling could not keep every graph's id range */
    bool rows_relabelled = true;
    /* nz row i: original vertex id, first edge position in col_r's order */
    dbuf<uint32_t> nz_rows, nz_start, zero_rows, head_bits, chunk_nz, od_nz;
    dbuf<uint4> split;
    uint32_t nlong = 0;
    dbuf<uint32_t> long_split; /* split rows spanning more than LONG_SPAN chunks */
    /* sources relabelled by out-degree (descending): col_r holds newid[col] of
     * the rows in plan order, each row's sources ascending */
    uint32_t hub = 0;
    dbuf<uint32_t> newid, col_r, nz_cidx, zero_cidx;
    /* launch configuration of the edge kernel (gcg_pagerank_autotune):
     * shared-memory hub entries (capped at hub) and chunks per warp run */
    uint32_t tune_hub = HUB_DEFAULT, tune_run = RUN_DEFAULT;
    /* sources relabelled within each interval (each interval keeps its id range) */
    bool per_interval = false;
};

/* builds (once per graph) the chunk plan and the out-degree relabelling */
int ensure_chunk_plan(gcg_graph *g);
/* builds (or keeps) the plan's source tiers for ntiers tiers of width ids */
int ensure_tier_plan(gcg_graph *g, int ntiers, uint32_t width);
int pr_init_state(gcg_graph *g, float init, const float *init_dev, float *r, float *c, float *rnz);

/* separate round-to-nearest multiply and add (no FMA contraction), as the
 * reference computes (float)(teleport + damping * (double)sum) */
__device__ __forceinline__ float pr_value(const SweepArgs &a, float sum) {
    return (float)__dadd_rn(a.teleport, __dmul_rn(a.damping, (double)sum));
}

}  // namespace gcg

#endif
