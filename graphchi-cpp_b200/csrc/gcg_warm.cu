/*
 * Learned warm start for PageRank: per-vertex degree features, a BF16 MLP
 * (8 -> 64 -> 64 -> 1), its training kernels and its tensor-core inference.
 *
 * No reference counterpart: the reference starts PageRank from a constant
 * (example_apps/pagerank.cpp:80-85) and has no learned component. The network
 * predicts y = log(rank / teleport); the Jacobi iteration started from
 * teleport * exp(y) then runs to the same residual as from the uniform start.
 *
 * Kernels
 *   k_warm_vstat   per vertex: {log(1+indeg), indeg} packed in 8 bytes, stored at
 *                  the vertex's out-degree rank (the PageRank relabelling)
 *   k_warm_agg_edges / k_warm_agg_fix   per vertex with in-edges: sum and max of
 *                  L(u) = log(1+indeg(u)) over in-neighbours u and the sum of
 *                  indeg(u), on the PageRank chunk plan: one warp per 256 in-edges
 *                  (edge-balanced whatever the degrees), one 8-byte gather per
 *                  edge (the 24576 highest out-degree sources from shared memory),
 *                  a warp segmented reduction of (sum, max, sum), rows crossing
 *                  chunks completed in chunk order
 *   k_warm_infer   the network on the 5th-generation tensor cores (tcgen05.mma,
 *                  BF16 operands in shared memory, FP32 accumulators in tensor
 *                  memory) over the vertices with in-edges (the others are set to
 *                  teleport): a CTA takes tiles of 128 vertices, layer 1 as one
 *                  M128 x N64 x K16 MMA (8 features padded to 16), layer 2 as four
 *                  K16 steps, each layer read back with tcgen05.ld; layer 3 and exp
 *                  on the FP32 pipes
 *   k_mlp_fwd_bwd  training: one sample per thread on the FP32 pipes (forward,
 *                  backward), then per-block weight gradients as small block
 *                  GEMMs over shared-memory activation tiles, one partial slot
 *                  per block (no atomics: the sum order is fixed)
 *   k_mlp_adam     fixed-order sum of the block partials, Adam on the FP32 master
 *                  weights, then the BF16-rounded copy the inference reads
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "gcg_internal.cuh"
#include "gcg_pr_device.cuh"

namespace gcg {
namespace {

constexpr int NIN = GCG_MLP_IN;
constexpr int NH = GCG_MLP_HIDDEN;
constexpr int NP = GCG_MLP_NPARAMS;
/* offsets in the flat parameter vector */
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH;
static_assert(OB3 + 1 == NP, "parameter layout");
constexpr int TRAIN_T = 128;        /* samples per training tile (one per thread) */
constexpr int HS = NH + 1;          /* padded row stride of the activation tiles */

/* round to the nearest BF16 value (ties to even), kept as a float */
__host__ __device__ __forceinline__ float bf16r(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}
__host__ __device__ __forceinline__ uint32_t bf16_bits(float x_rounded) {
    uint32_t u;
    memcpy(&u, &x_rounded, 4);
    return u >> 16;
}

/* ---- features ------------------------------------------------------------ */

/* The in-neighbourhood aggregates run on the PageRank chunk plan: 256-edge warp
 * chunks over the in-CSR with sources relabelled by out-degree, head bits for
 * row starts, split rows completed in chunk order. Each edge contributes
 * {L(u), L(u), indeg(u)} to its row's (sum, max, sum). */
struct AggArgs {
    const uint32_t *col; /* relabelled sources */
    const uint8_t *heads;
    const uint32_t *chunk_nz;
    uint64_t ne;
    uint32_t nchunks, hub;
    const uint2 *vstat; /* {L(u) as float bits, indeg(u)} by relabelled id */
};
struct AggOut {
    Agg3 *nzsum, *head_part, *tail_part;
};
constexpr uint32_t AGG_HUB_MAX = 24576; /* 192 KB of {L, indeg} pairs */

__global__ void k_warm_vstat(const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ newid, uint32_t nv,
                             uint2 *__restrict__ vstat) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t d = indeg[v];
        vstat[newid[v]] = make_uint2(__float_as_uint(log1pf((float)d)), d);
    }
}

__device__ __forceinline__ uint2 ld_keep_u2(const uint2 *p, uint64_t pol) {
    uint2 r;
    asm("ld.global.nc.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;" : "=r"(r.x), "=r"(r.y) : "l"(p), "l"(pol));
    return r;
}

__global__ void __launch_bounds__(EDGE_THREADS, 1) k_warm_agg_edges(AggArgs a, AggOut o) {
    extern __shared__ uint2 s_vs[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint64_t pol_stream = policy_evict_first(), pol_keep = policy_evict_last();
    for (uint32_t i = threadIdx.x; i < a.hub; i += blockDim.x) s_vs[i] = a.vstat[i];
    __syncthreads();
    uint32_t ch = gwarp;
    uint32_t col[EPL], flags = 0, nvalid = 0, base = 0;
    if (ch < a.nchunks) load_chunk(a, ch, lane, pol_stream, col, flags, nvalid, base, a.ne);
    for (; ch < a.nchunks; ch += nwarps) {
        Agg3 val[EPL];
#pragma unroll
        for (int j = 0; j < EPL; ++j) {
            const uint32_t x = col[j];
            uint2 w = make_uint2(0u, 0u);
            if ((uint32_t)j < nvalid) w = x < a.hub ? s_vs[x] : ld_keep_u2(a.vstat + x, pol_keep);
            const float L = __uint_as_float(w.x);
            val[j] = Agg3{L, L, (float)w.y};
        }
        const uint32_t cf = flags, cn = nvalid, cb = base;
        if (ch + nwarps < a.nchunks) load_chunk(a, ch + nwarps, lane, pol_stream, col, flags, nvalid, base, a.ne);
        reduce_chunk_to(a, o, ch, lane, val, cf, cn, cb, a.ne);
    }
}

/* rows crossing chunks, in chunk order (the order of the PageRank fix-up): the
 * long ones (more than LONG_SPAN chunks; rows in relabelled order put them next to each
 * other) one per warp over the grid, lane-strided partials reduced by an xor
 * tree; the others one per lane */
__global__ void __launch_bounds__(256) k_warm_agg_fix(const uint4 *__restrict__ split, uint32_t nsplit,
                                                      const uint32_t *__restrict__ long_split, uint32_t nlong,
                                                      AggOut o) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = gwarp; r < nlong; r += nwarps) {
        const uint4 sp = split[long_split[r]];
        Agg3 v = Agg3{0.0f, 0.0f, 0.0f};
        for (uint32_t c = sp.y + 1 + lane; c <= sp.z; c += 32u) v = vadd(v, o.head_part[c]);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
            v = vadd(v, Agg3{__shfl_xor_sync(FULL, v.s, d), __shfl_xor_sync(FULL, v.m, d),
                             __shfl_xor_sync(FULL, v.t, d)});
        if (lane == 0) o.nzsum[sp.x] = vadd(o.tail_part[sp.y], v);
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nsplit; k += gridDim.x * blockDim.x) {
        const uint4 sp = split[k];
        if (sp.z - sp.y <= LONG_SPAN) {
            Agg3 v = o.tail_part[sp.y];
            for (uint32_t c = sp.y + 1; c <= sp.z; ++c) v = vadd(v, o.head_part[c]);
            o.nzsum[sp.x] = v;
        }
    }
}

/* raw feature k of vertex v (ag: its in-neighbourhood aggregates; zero without in-edges) */
__device__ __forceinline__ float feature(int k, uint32_t v, uint32_t din, uint32_t dout, Agg3 ag, uint32_t vbits) {
    switch (k) {
        case 0: return log1pf((float)din);
        case 1: return log1pf((float)dout);
        case 2: return din ? ag.s / (float)din : 0.0f;
        case 3: return din ? ag.m : 0.0f;
        case 4: return din ? log1pf(ag.t) : 0.0f;
        case 5: return dout ? 1.0f / (float)dout : 0.0f;
        case 6: return vbits >= 1 ? (float)((v >> (vbits - 1)) & 1u) : 0.0f;
        default: return vbits >= 2 ? (float)((v >> (vbits - 2)) & 1u) : 0.0f;
    }
}

/* features of every vertex: nz rows from the aggregates, the others without */
__global__ void k_warm_features(const uint32_t *__restrict__ nz_rows, uint32_t nnz,
                                const uint32_t *__restrict__ zero_rows, uint32_t nzero,
                                const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ outdeg,
                                const Agg3 *__restrict__ agg, uint32_t vbits, float *__restrict__ out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < nnz + nzero; i += nth) {
        const bool nz = i < nnz;
        const uint32_t v = nz ? nz_rows[i] : zero_rows[i - nnz];
        const Agg3 ag = nz ? agg[i] : Agg3{0.0f, 0.0f, 0.0f};
        const uint32_t din = nz ? indeg[v] : 0u, dout = outdeg[v];
#pragma unroll
        for (int k = 0; k < NIN; ++k) out[(size_t)v * NIN + k] = feature(k, v, din, dout, ag, vbits);
    }
}

/* ---- inference on tensor cores ------------------------------------------ */

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    return bf16_bits(lo) | (bf16_bits(hi) << 16);
}

/* normalised BF16 inputs of the vertices with in-edges, 16 bytes per row:
 * word t holds features 2t and 2t+1, i.e. the row exactly as the first K core
 * matrix of the inference's A tile holds it */
__global__ void k_warm_xfeat(const uint32_t *__restrict__ nz_rows, const uint32_t *__restrict__ od_nz, uint32_t nnz,
                             const uint32_t *__restrict__ indeg, const Agg3 *__restrict__ agg, uint32_t vbits,
                             const float *__restrict__ norm, uint4 *__restrict__ xpk) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        const uint32_t v = nz_rows[i], din = indeg[v], dout = od_nz[i];
        const Agg3 ag = agg[i];
        uint32_t w[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float f0 = (feature(2 * t, v, din, dout, ag, vbits) - norm[2 * t]) * norm[NIN + 2 * t];
            const float f1 = (feature(2 * t + 1, v, din, dout, ag, vbits) - norm[2 * t + 1]) * norm[NIN + 2 * t + 1];
            w[t] = pack_bf16(bf16r(f0), bf16r(f1));
        }
        xpk[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

/* ---- inference on the 5th-generation tensor cores (tcgen05) -------------
 * One CTA of 128 threads takes tiles of 128 vertices with in-edges (one row per
 * thread). Both layers are tcgen05.mma of kind f16 (BF16 operands, FP32
 * accumulation) with M = 128, N = 64, issued by one thread: layer 1 is one MMA
 * (K = 16: the 8 features and 8 zero columns), layer 2 four (K = 64). The
 * operands sit in shared memory as K-major "core matrices" without swizzle (8
 * rows x 16 bytes each, contiguous); the accumulator is a 128-lane x 64-column
 * FP32 tile in tensor memory, read back with tcgen05.ld (warp w reads lanes
 * 32w..32w+31, so every thread receives its own row). Each layer's completion
 * is signalled on an mbarrier by tcgen05.commit; every wait is bounded. */
constexpr int TC_ROWS = 128;   /* M of the MMA: rows of a tile, threads of a CTA */
constexpr int TC_COLS = 64;    /* tensor-memory columns held by a CTA (the N of both layers) */
constexpr uint32_t TC_CTAS_PER_SM = 4;
/* instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
 * (bits 7-9 = 1) and B (bits 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3
 * in bits 17-22, M >> 4 in bits 24-28 */
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NH >> 3) << 17) |
                              ((uint32_t)(TC_ROWS >> 4) << 24);

/* shared-memory matrix descriptor, no swizzle: start address, the byte offset
 * between the two K-adjacent core matrices (lbo) and between 8-row groups (sbo),
 * all in 16-byte units; descriptor version 1 (bit 46) */
__device__ __forceinline__ uint64_t tc_desc(const void *smem, uint32_t lbo, uint32_t sbo) {
    const uint32_t a = smem_u32(smem);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate)
        : "memory");
}
/* arrives once on bar when every MMA this thread issued before has completed */
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
/* generic-proxy writes to shared memory become visible to the tensor cores */
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
/* 16 consecutive FP32 columns of this thread's tensor-memory lane */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
/* byte offset of element (row, k) in a K-major core-matrix tile whose rows have
 * kcores cores of 8 BF16 */
__host__ __device__ __forceinline__ uint32_t tc_off(uint32_t row, uint32_t k, uint32_t kcores) {
    return ((row >> 3) * kcores + (k >> 3)) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

struct InferArgs {
    const uint32_t *nz_rows, *od_nz;
    const uint4 *xpk;              /* per nz row: 8 normalised BF16 features */
    uint32_t nnz;
    const float *wb;               /* BF16-rounded weights, FP32 biases */
    float teleport;
    float *out;
    double2 *part_mass;            /* per block: sum of the predicted ranks, of those without out-edges */
    int *err;                      /* set when a wait for the tensor cores ran out */
};

__global__ void __launch_bounds__(TC_ROWS) k_warm_infer(InferArgs a) {
    __shared__ __align__(1024) uint8_t s_a1[TC_ROWS * 16 * 2]; /* X: 128 x 16 BF16 */
    __shared__ __align__(1024) uint8_t s_b1[NH * 16 * 2];      /* W1: 64 x 16 BF16 */
    __shared__ __align__(1024) uint8_t s_a2[TC_ROWS * NH * 2]; /* H1: 128 x 64 BF16 */
    __shared__ __align__(1024) uint8_t s_b2[NH * NH * 2];      /* W2: 64 x 64 BF16 */
    __shared__ float s_bias1[NH], s_bias2[NH], s_w3[NH];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ double s_m[TC_ROWS / 32][2];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;

    /* weights into the K-major core-matrix layout (layer 1 padded to K = 16) */
    for (uint32_t e = tid; e < (uint32_t)NH * 16; e += TC_ROWS) {
        const uint32_t n = e >> 4, k = e & 15u;
        const float w = k < (uint32_t)NIN ? a.wb[OW1 + n * NIN + k] : 0.0f;
        *(uint16_t *)(s_b1 + tc_off(n, k, 2)) = (uint16_t)bf16_bits(w);
    }
    for (uint32_t e = tid; e < (uint32_t)NH * NH; e += TC_ROWS) {
        const uint32_t n = e >> 6, k = e & 63u;
        *(uint16_t *)(s_b2 + tc_off(n, k, NH / 8)) = (uint16_t)bf16_bits(a.wb[OW2 + n * NH + k]);
    }
    for (uint32_t j = tid; j < (uint32_t)NH; j += TC_ROWS) {
        s_bias1[j] = a.wb[OB1 + j];
        s_bias2[j] = a.wb[OB2 + j];
        s_w3[j] = a.wb[OW3 + j];
    }
    /* the zero K-columns 8..15 of every X row */
    *(uint4 *)(s_a1 + tc_off(tid, 8, 2)) = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        s_fail = 0;
        mbar_init(&s_bar, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"((uint32_t)TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t taddr = tmem + ((warp * 32u) << 16); /* this warp's 32 lanes */
    const float b3 = a.wb[OB3];
    const uint64_t d_a1 = tc_desc(s_a1, 128, 256), d_b1 = tc_desc(s_b1, 128, 256);

    double msum = 0.0, mdang = 0.0;
    uint32_t phase = 0;
    const uint32_t ntiles = (a.nnz + TC_ROWS - 1) / TC_ROWS;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t i = tile * TC_ROWS + tid;
        const bool valid = i < a.nnz;
        const uint4 x = valid ? a.xpk[i] : make_uint4(0u, 0u, 0u, 0u);
        const uint32_t v = valid ? a.nz_rows[i] : 0u, od = valid ? a.od_nz[i] : 1u;
        *(uint4 *)(s_a1 + tc_off(tid, 0, 2)) = x;
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (s_fail) break; /* a wait of the previous tile ran out (uniform: read after the barrier) */
        tc_fence_after();
        if (tid == 0) {
            tc_mma(tmem, d_a1, d_b1, 0u);
            tc_commit(&s_bar);
        }
        bool ok = false;
        for (long long spin = 0; !ok && spin < MBAR_SPIN; ++spin) ok = mbar_try_wait(&s_bar, phase);
        phase ^= 1u;
        if (!ok) s_fail = 1;
        tc_fence_after();
        float acc[NH];
#pragma unroll
        for (int q = 0; q < NH / 16; ++q) tc_ld16(taddr + 16u * q, acc + 16 * q);
        tc_wait_ld();
        /* layer-1 epilogue: bias, ReLU, BF16, into this thread's row of H1 */
#pragma unroll
        for (int kc = 0; kc < NH / 8; ++kc) {
            uint32_t w[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int j = kc * 8 + 2 * t;
                const float h0 = bf16r(fmaxf(acc[j] + s_bias1[j], 0.0f));
                const float h1 = bf16r(fmaxf(acc[j + 1] + s_bias1[j + 1], 0.0f));
                w[t] = bf16_bits(h0) | (bf16_bits(h1) << 16);
            }
            *(uint4 *)(s_a2 + tc_off(tid, kc * 8, NH / 8)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (s_fail) break;
        tc_fence_after();
        if (tid == 0) {
#pragma unroll
            for (int st = 0; st < NH / 16; ++st)
                tc_mma(tmem, tc_desc(s_a2 + 256 * st, 128, 1024), tc_desc(s_b2 + 256 * st, 128, 1024), st > 0);
            tc_commit(&s_bar);
        }
        ok = false;
        for (long long spin = 0; !ok && spin < MBAR_SPIN; ++spin) ok = mbar_try_wait(&s_bar, phase);
        phase ^= 1u;
        if (!ok) s_fail = 1;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < NH / 16; ++q) tc_ld16(taddr + 16u * q, acc + 16 * q);
        tc_wait_ld();
        /* layer 2's bias and ReLU, layer 3 on the FP32 pipes */
        float y = 0.0f;
#pragma unroll
        for (int j = 0; j < NH; ++j) y = fmaf(fmaxf(acc[j] + s_bias2[j], 0.0f), s_w3[j], y);
        if (valid) {
            /* y is clamped so exp stays finite */
            const float r = a.teleport * expf(fminf(fmaxf(y + b3, -30.0f), 30.0f));
            a.out[v] = r;
            msum += (double)r;
            if (od == 0) mdang += (double)r;
        }
        tc_fence_before(); /* this tile's tensor-memory reads precede the next tile's MMA */
    }
    __syncthreads();
    if (tid == 0 && s_fail) atomicExch(a.err, 1);
    /* block partials of the mass terms, reduced in a fixed order */
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        msum += __shfl_xor_sync(0xFFFFFFFFu, msum, o);
        mdang += __shfl_xor_sync(0xFFFFFFFFu, mdang, o);
    }
    if (lane == 0) {
        s_m[warp][0] = msum;
        s_m[warp][1] = mdang;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
        double2 m = make_double2(0.0, 0.0);
        for (int w = 0; w < TC_ROWS / 32; ++w) {
            m.x += s_m[w][0];
            m.y += s_m[w][1];
        }
        a.part_mass[blockIdx.x] = m;
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_COLS)
                     : "memory");
}

/* vertices without in-edges: exactly teleport; per block, how many also lack out-edges */
__global__ void __launch_bounds__(256) k_warm_zero(const uint32_t *__restrict__ zero_rows, uint32_t nzero,
                                                   const uint32_t *__restrict__ outdeg, float teleport,
                                                   float *__restrict__ out, uint32_t *__restrict__ part_zd) {
    __shared__ uint32_t s_c[8];
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nzero; i += gridDim.x * blockDim.x) {
        const uint32_t v = zero_rows[i];
        out[v] = teleport;
        c += outdeg[v] == 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31u) == 0) s_c[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_c[w];
        part_zd[blockIdx.x] = tot;
    }
}

/* Mass-stationary scale of the predicted ranks: alpha such that one Jacobi sweep
 * keeps the total rank. With Z = vertices without in-edges (rank = teleport
 * exactly), D = vertices without out-edges, M = sum of the predictions outside Z
 * and M_D = the part of M on D, the sweep's total is teleport*n +
 * damping*(total - total on D), which equals the total when
 *   alpha = teleport*(n - (1-damping)|Z| - damping|Z & D|) / ((1-damping)M + damping M_D). */
__global__ void k_warm_alpha(const double2 *__restrict__ pm, uint32_t nmass, const uint32_t *__restrict__ pzd,
                             uint32_t nzd, uint32_t nv, uint32_t nzero, double teleport, double damping,
                             double *__restrict__ alpha) {
    const uint32_t lane = threadIdx.x;
    double M = 0.0, MD = 0.0;
    unsigned long long zd = 0;
    for (uint32_t b = lane; b < nmass; b += 32u) {
        M += pm[b].x;
        MD += pm[b].y;
    }
    for (uint32_t b = lane; b < nzd; b += 32u) zd += pzd[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        M += __shfl_xor_sync(0xFFFFFFFFu, M, o);
        MD += __shfl_xor_sync(0xFFFFFFFFu, MD, o);
        zd += __shfl_xor_sync(0xFFFFFFFFu, zd, o);
    }
    if (lane == 0) {
        const double den = (1.0 - damping) * M + damping * MD;
        const double num = teleport * ((double)nv - (1.0 - damping) * (double)nzero - damping * (double)zd);
        *alpha = (den > 0.0 && num > 0.0) ? num / den : 1.0;
    }
}

__global__ void k_warm_scale(const uint32_t *__restrict__ nz_rows, uint32_t nnz, const double *__restrict__ alpha,
                             float *__restrict__ out) {
    const double al = *alpha;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        const uint32_t v = nz_rows[i];
        out[v] = (float)((double)out[v] * al);
    }
}

/* ---- training -------------------------------------------------------------- */

struct TrainArgs {
    const float *x, *t;     /* samples: x [n][8] raw features, t [n] targets */
    const uint32_t *idx;    /* sample order (NULL = identity) */
    uint64_t base, count;   /* this batch: positions [base, base + count) of the order */
    const float *wb;        /* rounded weights, FP32 biases */
    const float *norm;      /* mean[8], inv_std[8] */
    float dscale;           /* dL/dy = dscale * (y - t): 2 / batch size */
    float *part;            /* [gridDim.x][NP + 1] gradient partials, last = sum of squared errors */
    float *yout;            /* forward only: y per sample of the batch */
};

/* shared-memory layout (floats) */
constexpr int SM_W = 0;                       /* rounded parameters [NP] */
constexpr int SM_H1 = (NP + 3) & ~3;          /* h1 [TRAIN_T][HS] */
constexpr int SM_H2 = SM_H1 + TRAIN_T * HS;   /* h2 */
constexpr int SM_D2 = SM_H2 + TRAIN_T * HS;   /* dL/da2 */
constexpr int SM_D1 = SM_D2 + TRAIN_T * HS;   /* dL/da1 */
constexpr int SM_X = SM_D1 + TRAIN_T * HS;    /* normalised inputs [TRAIN_T][8] */
constexpr int SM_DY = SM_X + TRAIN_T * NIN;   /* dL/dy [TRAIN_T] */
constexpr int SM_RED = SM_DY + TRAIN_T;       /* loss reduction [TRAIN_T] */
constexpr int SM_TOTAL = SM_RED + TRAIN_T;
constexpr size_t TRAIN_SMEM = (size_t)SM_TOTAL * 4;

/* Forward (and, with FWD_ONLY false, backward) of one training tile per
 * iteration: thread s runs sample s through the network on the FP32 pipes; the
 * weight gradients are then accumulated as block GEMMs over the tile's
 * activations: thread p owns row j = p/2 of dW2 (32 columns), of dW1 (4 columns)
 * and one bias or W3 entry. */
template <bool FWD_ONLY>
__global__ void __launch_bounds__(TRAIN_T) k_mlp_fwd_bwd(TrainArgs a) {
    extern __shared__ float sm[];
    float *sw = sm + SM_W, *sH1 = sm + SM_H1, *sH2 = sm + SM_H2, *sD2 = sm + SM_D2, *sD1 = sm + SM_D1,
          *sX = sm + SM_X, *sDy = sm + SM_DY, *sRed = sm + SM_RED;
    for (int i = threadIdx.x; i < NP; i += TRAIN_T) sw[i] = a.wb[i];
    __syncthreads();
    const float *W1 = sw + OW1, *B1 = sw + OB1, *W2 = sw + OW2, *B2 = sw + OB2, *W3 = sw + OW3;
    const float b3 = sw[OB3];
    const uint32_t s = threadIdx.x, p = threadIdx.x, jj = p >> 1, half = p & 1u;
    float gW2[32], gW1[4], gA = 0.0f, gB = 0.0f, gb3 = 0.0f, loss = 0.0f;
#pragma unroll
    for (int k = 0; k < 32; ++k) gW2[k] = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) gW1[q] = 0.0f;
    const uint64_t ntiles = (a.count + TRAIN_T - 1) / TRAIN_T;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t i = tile * TRAIN_T + s;
        const bool valid = i < a.count;
        uint64_t row = 0;
        if (valid) row = a.idx ? a.idx[a.base + i] : a.base + i;
        float xh[NIN];
#pragma unroll
        for (int k = 0; k < NIN; ++k)
            xh[k] = valid ? bf16r((a.x[row * NIN + k] - a.norm[k]) * a.norm[NIN + k]) : 0.0f;
        /* layer 1 */
        float h[NH];
        uint64_t m1 = 0, m2 = 0;
#pragma unroll
        for (int j = 0; j < NH; ++j) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < NIN; ++k) acc = fmaf(W1[j * NIN + k], xh[k], acc);
            acc += B1[j];
            if (acc > 0.0f) m1 |= 1ull << j;
            h[j] = bf16r(fmaxf(acc, 0.0f));
            sH1[s * HS + j] = h[j];
        }
        /* layers 2 and 3 */
        float y = 0.0f;
        for (int j = 0; j < NH; ++j) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < NH; ++k) acc = fmaf(W2[j * NH + k], h[k], acc);
            acc += B2[j];
            if (acc > 0.0f) m2 |= 1ull << j;
            const float h2 = fmaxf(acc, 0.0f);
            sH2[s * HS + j] = h2;
            y = fmaf(W3[j], h2, y);
        }
        y += b3;
        if (FWD_ONLY) {
            if (valid) a.yout[i] = y;
            continue;
        }
        const float err = valid ? y - a.t[row] : 0.0f;
        loss = fmaf(err, err, loss);
        const float dy = a.dscale * err;
        sDy[s] = dy;
#pragma unroll
        for (int k = 0; k < NIN; ++k) sX[s * NIN + k] = xh[k];
        /* backward through layers 3 and 2 (h is reused for dL/dh1) */
#pragma unroll
        for (int k = 0; k < NH; ++k) h[k] = 0.0f;
        for (int j = 0; j < NH; ++j) {
            const float d2 = ((m2 >> j) & 1ull) ? dy * W3[j] : 0.0f;
            sD2[s * HS + j] = d2;
#pragma unroll
            for (int k = 0; k < NH; ++k) h[k] = fmaf(W2[j * NH + k], d2, h[k]);
        }
#pragma unroll
        for (int k = 0; k < NH; ++k) sD1[s * HS + k] = ((m1 >> k) & 1ull) ? h[k] : 0.0f;
        __syncthreads();
        /* weight gradients over the tile's samples, in sample order */
        for (int q = 0; q < TRAIN_T; ++q) {
            const float d2 = sD2[q * HS + jj], d1 = sD1[q * HS + jj];
            const float *h1 = sH1 + q * HS + half * 32;
#pragma unroll
            for (int k = 0; k < 32; ++k) gW2[k] = fmaf(d2, h1[k], gW2[k]);
            const float *xq = sX + q * NIN + half * 4;
#pragma unroll
            for (int k = 0; k < 4; ++k) gW1[k] = fmaf(d1, xq[k], gW1[k]);
            if (half == 0) {
                gA += d2;                                  /* db2[jj] */
                gB = fmaf(sDy[q], sH2[q * HS + jj], gB);   /* dW3[jj] */
            } else {
                gA += d1;                                  /* db1[jj] */
                if (p == 1) gb3 += sDy[q];
            }
        }
        __syncthreads();
    }
    if (FWD_ONLY) return;
    float *out = a.part + (size_t)blockIdx.x * (NP + 1);
#pragma unroll
    for (int k = 0; k < 32; ++k) out[OW2 + jj * NH + half * 32 + k] = gW2[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) out[OW1 + jj * NIN + half * 4 + k] = gW1[k];
    if (half == 0) {
        out[OB2 + jj] = gA;
        out[OW3 + jj] = gB;
    } else {
        out[OB1 + jj] = gA;
        if (p == 1) out[OB3] = gb3;
    }
    /* sum of squared errors: fixed tree over the block */
    sRed[p] = loss;
    __syncthreads();
    for (int w = TRAIN_T / 2; w > 0; w >>= 1) {
        if ((int)p < w) sRed[p] += sRed[p + w];
        __syncthreads();
    }
    if (p == 0) out[NP] = sRed[0];
}

struct AdamArgs {
    const float *part;
    uint32_t nblocks;
    float *w, *wb, *m, *v;
    float lr, beta1, beta2, eps, bc1, bc2; /* bc = 1 - beta^step */
    int apply;
    float *grad_out;   /* optional: the summed gradient */
    double *loss_acc;  /* optional: += sum of squared errors */
};

__device__ __forceinline__ bool is_weight(int i) {
    return i < OB1 || (i >= OW2 && i < OB2) || (i >= OW3 && i < OB3);
}

__global__ void k_mlp_adam(AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < NP) {
        float gsum = 0.0f;
        for (uint32_t b = 0; b < a.nblocks; ++b) gsum += a.part[(size_t)b * (NP + 1) + i];
        if (a.grad_out) a.grad_out[i] = gsum;
        if (a.apply) {
            const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * gsum;
            const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * gsum * gsum;
            a.m[i] = m;
            a.v[i] = v;
            const float w = a.w[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
            a.w[i] = w;
            a.wb[i] = is_weight(i) ? bf16r(w) : w;
        }
    } else if (i == NP && a.loss_acc) {
        double l = 0.0;
        for (uint32_t b = 0; b < a.nblocks; ++b) l += (double)a.part[(size_t)b * (NP + 1) + NP];
        *a.loss_acc += l;
    }
}

__global__ void k_mlp_round(const float *__restrict__ w, float *__restrict__ wb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x)
        wb[i] = is_weight(i) ? bf16r(w[i]) : w[i];
}

}  // namespace
}  // namespace gcg

/* ---- host side ------------------------------------------------------------- */

struct gcg_mlp {
    gcg::dbuf<float> w, wb, m, v, norm; /* master weights, rounded copy, Adam moments, normalisation */
    uint64_t step = 0;                  /* Adam steps taken */
};

namespace gcg {
namespace {

uint64_t splitmix(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t &x) { return ((splitmix(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

/* rounded copy of the master weights (stream-ordered) */
int mlp_prepare(gcg_mlp *m, cudaStream_t s) {
    k_mlp_round<<<(NP + 255) / 256, 256, 0, s>>>(m->w.get(), m->wb.get());
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

/* device copy of a user array (host or device) of n elements */
template <typename T>
int stage_in(const T *user, size_t n, tbuf<T> &tmp, const T **dev, cudaStream_t s) {
    if (is_device_ptr(user)) {
        *dev = user;
        return GCG_OK;
    }
    GCG_TRY(tmp.alloc(n, s));
    GCG_TRY(copy_in(tmp.get(), user, n * sizeof(T), s));
    *dev = tmp.get();
    return GCG_OK;
}

int train_grid(uint64_t count) {
    const uint64_t ntiles = (count + TRAIN_T - 1) / TRAIN_T;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(ntiles, (uint64_t)num_sms()));
}

int set_train_smem() {
    GCG_CUDA(cudaFuncSetAttribute(k_mlp_fwd_bwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
    GCG_CUDA(cudaFuncSetAttribute(k_mlp_fwd_bwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
    return GCG_OK;
}

/* per-nz-row aggregates of the in-neighbourhood (features 2-4), on the chunk plan */
int warm_aggregates(gcg_graph *g, tbuf<Agg3> &agg, cudaStream_t s) {
    GCG_TRY(ensure_chunk_plan(g));
    const ChunkPlan &pl = *g->cplan;
    const uint32_t nv = g->nv;
    tbuf<uint2> vstat;
    tbuf<Agg3> parts;
    GCG_TRY(vstat.alloc(nv, s));
    GCG_TRY(agg.alloc(std::max<uint32_t>(pl.nnz, 1), s));
    GCG_TRY(parts.alloc((size_t)2 * pl.nchunks + 2, s));
    const int sms = num_sms();
    const unsigned b1 = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, sms * 8ull));
    k_warm_vstat<<<b1, 256, 0, s>>>(g->indeg.get(), pl.newid.get(), nv, vstat.get());
    if (pl.nchunks) {
        AggArgs a;
        a.col = pl.col_r.get();
        a.heads = (const uint8_t *)pl.head_bits.get();
        a.chunk_nz = pl.chunk_nz.get();
        a.ne = g->ne;
        a.nchunks = pl.nchunks;
        a.hub = std::min<uint32_t>(nv, AGG_HUB_MAX);
        a.vstat = vstat.get();
        AggOut o;
        o.nzsum = agg.get();
        o.head_part = parts.get();
        o.tail_part = parts.get() + pl.nchunks + 1;
        const size_t smem = (size_t)AGG_HUB_MAX * sizeof(uint2);
        GCG_CUDA(cudaFuncSetAttribute(k_warm_agg_edges, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const unsigned grid = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>(((uint64_t)pl.nchunks * 32 + EDGE_THREADS - 1) / EDGE_THREADS, (uint64_t)sms));
        k_warm_agg_edges<<<grid, EDGE_THREADS, (size_t)a.hub * sizeof(uint2), s>>>(a, o);
        if (pl.nsplit) {
            const unsigned fb = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>(((uint64_t)pl.nsplit + 255) / 256, sms * 8ull));
            k_warm_agg_fix<<<fb, 256, 0, s>>>(pl.split.get(), pl.nsplit, pl.long_split.get(), pl.nlong, o);
        }
    }
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

}  // namespace
}  // namespace gcg

using namespace gcg;

extern "C" {

int gcg_mlp_create(uint64_t seed, gcg_mlp **out) {
    if (!out) return fail(GCG_ERR_INVALID, "gcg_mlp_create: null output");
    *out = nullptr;
    gcg_mlp *m = new gcg_mlp();
    std::vector<float> w(NP, 0.0f), zero(NP, 0.0f), norm(2 * NIN, 0.0f);
    uint64_t st = seed ^ 0x5EEDC0DEull;
    auto normal = [&](double sd) {
        const double u1 = uniform01(st), u2 = uniform01(st);
        return (float)(sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
    };
    for (int i = 0; i < NH * NIN; ++i) w[OW1 + i] = normal(sqrt(2.0 / NIN));
    for (int i = 0; i < NH * NH; ++i) w[OW2 + i] = normal(sqrt(2.0 / NH));
    for (int i = 0; i < NH; ++i) w[OW3 + i] = normal(sqrt(1.0 / NH));
    for (int i = 0; i < NIN; ++i) norm[NIN + i] = 1.0f;
    int rc;
    if ((rc = m->w.alloc(NP)) || (rc = m->wb.alloc(NP)) || (rc = m->m.alloc(NP)) || (rc = m->v.alloc(NP)) ||
        (rc = m->norm.alloc(2 * NIN))) {
        delete m;
        return rc;
    }
    cudaError_t e = cudaMemcpy(m->w.get(), w.data(), NP * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->m.get(), zero.data(), NP * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->v.get(), zero.data(), NP * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->norm.get(), norm.data(), 2 * NIN * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete m;
        return fail(GCG_ERR_CUDA, std::string("gcg_mlp_create: ") + cudaGetErrorString(e));
    }
    if ((rc = mlp_prepare(m, 0)) != GCG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return GCG_OK;
}

int gcg_mlp_free(gcg_mlp *m) {
    if (m) {
        cudaDeviceSynchronize();
        delete m;
    }
    return GCG_OK;
}

int gcg_mlp_get(const gcg_mlp *m, float *params, float *norm) {
    if (!m) return fail(GCG_ERR_INVALID, "gcg_mlp_get: null model");
    GCG_CUDA(cudaDeviceSynchronize());
    if (params) GCG_CUDA(cudaMemcpy(params, m->w.get(), NP * 4, cudaMemcpyDefault));
    if (norm) GCG_CUDA(cudaMemcpy(norm, m->norm.get(), 2 * NIN * 4, cudaMemcpyDefault));
    return GCG_OK;
}

int gcg_mlp_set(gcg_mlp *m, const float *params, const float *norm) {
    if (!m) return fail(GCG_ERR_INVALID, "gcg_mlp_set: null model");
    GCG_CUDA(cudaDeviceSynchronize());
    if (params) {
        std::vector<float> zero(NP, 0.0f);
        GCG_CUDA(cudaMemcpy(m->w.get(), params, NP * 4, cudaMemcpyDefault));
        GCG_CUDA(cudaMemcpy(m->m.get(), zero.data(), NP * 4, cudaMemcpyHostToDevice));
        GCG_CUDA(cudaMemcpy(m->v.get(), zero.data(), NP * 4, cudaMemcpyHostToDevice));
        m->step = 0;
    }
    if (norm) GCG_CUDA(cudaMemcpy(m->norm.get(), norm, 2 * NIN * 4, cudaMemcpyDefault));
    GCG_TRY(mlp_prepare(m, 0));
    GCG_CUDA(cudaDeviceSynchronize());
    return GCG_OK;
}

int gcg_mlp_fit_normalisation(gcg_mlp *m, const float *x, uint64_t n) {
    if (!m || !x || n == 0) return fail(GCG_ERR_INVALID, "gcg_mlp_fit_normalisation: bad argument");
    std::vector<float> h((size_t)n * NIN);
    GCG_CUDA(cudaMemcpy(h.data(), x, h.size() * 4, cudaMemcpyDefault));
    double mu[NIN] = {0}, sq[NIN] = {0};
    for (uint64_t i = 0; i < n; ++i)
        for (int k = 0; k < NIN; ++k) mu[k] += h[i * NIN + k];
    for (int k = 0; k < NIN; ++k) mu[k] /= (double)n;
    for (uint64_t i = 0; i < n; ++i)
        for (int k = 0; k < NIN; ++k) {
            const double d = h[i * NIN + k] - mu[k];
            sq[k] += d * d;
        }
    float norm[2 * NIN];
    for (int k = 0; k < NIN; ++k) {
        const double sd = sqrt(sq[k] / (double)n);
        norm[k] = (float)mu[k];
        norm[NIN + k] = sd > 1e-12 ? (float)(1.0 / sd) : 1.0f;
    }
    GCG_CUDA(cudaMemcpy(m->norm.get(), norm, sizeof(norm), cudaMemcpyHostToDevice));
    return GCG_OK;
}

int gcg_warm_features(gcg_graph *g, float *features) {
    if (!g || !features) return fail(GCG_ERR_INVALID, "gcg_warm_features: null argument");
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    tbuf<Agg3> agg;
    GCG_TRY(warm_aggregates(g, agg, s));
    const ChunkPlan &pl = *g->cplan;
    tbuf<float> stage;
    float *dst = features;
    const bool dev = is_device_ptr(features);
    if (!dev) {
        GCG_TRY(stage.alloc((size_t)nv * NIN, s));
        dst = stage.get();
    }
    const unsigned b = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, num_sms() * 8ull));
    k_warm_features<<<b, 256, 0, s>>>(pl.nz_rows.get(), pl.nnz, pl.zero_rows.get(), pl.nzero, g->indeg.get(),
                                      g->outdeg.get(), agg.get(), g->vbits, dst);
    GCG_LAUNCH_CHECK();
    if (!dev) GCG_TRY(copy_out(features, dst, (size_t)nv * NIN * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

int gcg_mlp_forward(const gcg_mlp *m, const float *x, uint64_t n, float *y) {
    if (!m || !x || !y) return fail(GCG_ERR_INVALID, "gcg_mlp_forward: null argument");
    if (n == 0) return GCG_OK;
    cudaStream_t s = 0;
    GCG_TRY(set_train_smem());
    tbuf<float> xs, ys;
    const float *xd;
    GCG_TRY(stage_in(x, (size_t)n * NIN, xs, &xd, s));
    float *yd = y;
    const bool dev = is_device_ptr(y);
    if (!dev) {
        GCG_TRY(ys.alloc(n, s));
        yd = ys.get();
    }
    TrainArgs a;
    memset(&a, 0, sizeof(a));
    a.x = xd;
    a.count = n;
    a.wb = m->wb.get();
    a.norm = m->norm.get();
    a.yout = yd;
    k_mlp_fwd_bwd<true><<<train_grid(n), TRAIN_T, TRAIN_SMEM, s>>>(a);
    GCG_LAUNCH_CHECK();
    if (!dev) GCG_TRY(copy_out(y, yd, (size_t)n * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

int gcg_mlp_gradient(const gcg_mlp *m, const float *x, const float *t, uint64_t n, float *grad, double *loss) {
    if (!m || !x || !t || n == 0) return fail(GCG_ERR_INVALID, "gcg_mlp_gradient: bad argument");
    cudaStream_t s = 0;
    GCG_TRY(set_train_smem());
    tbuf<float> xs, ts, part, gd;
    tbuf<double> acc;
    const float *xd, *td;
    GCG_TRY(stage_in(x, (size_t)n * NIN, xs, &xd, s));
    GCG_TRY(stage_in(t, (size_t)n, ts, &td, s));
    const int grid = train_grid(n);
    GCG_TRY(part.alloc((size_t)grid * (NP + 1), s));
    GCG_TRY(gd.alloc(NP, s));
    GCG_TRY(acc.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(acc.get(), 0, 8, s));
    TrainArgs a;
    memset(&a, 0, sizeof(a));
    a.x = xd;
    a.t = td;
    a.count = n;
    a.wb = m->wb.get();
    a.norm = m->norm.get();
    a.dscale = (float)(2.0 / (double)n);
    a.part = part.get();
    k_mlp_fwd_bwd<false><<<grid, TRAIN_T, TRAIN_SMEM, s>>>(a);
    AdamArgs d;
    memset(&d, 0, sizeof(d));
    d.part = part.get();
    d.nblocks = (uint32_t)grid;
    d.apply = 0;
    d.grad_out = gd.get();
    d.loss_acc = acc.get();
    k_mlp_adam<<<(NP + 1 + 255) / 256, 256, 0, s>>>(d);
    GCG_LAUNCH_CHECK();
    double l = 0.0;
    GCG_CUDA(cudaMemcpyAsync(&l, acc.get(), 8, cudaMemcpyDeviceToHost, s));
    if (grad) GCG_TRY(copy_out(grad, gd.get(), NP * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l / (double)n;
    return GCG_OK;
}

void gcg_mlp_train_params_default(gcg_mlp_train_params *p) {
    if (!p) return;
    p->epochs = 8;
    p->batch = 4096;
    p->lr = 2e-3f;
    p->beta1 = 0.9f;
    p->beta2 = 0.999f;
    p->eps = 1e-8f;
    p->seed = 1;
}

int gcg_mlp_train(gcg_mlp *m, const float *x, const float *t, uint64_t n, const gcg_mlp_train_params *p,
                  float *epoch_loss) {
    if (!m || !x || !t || !p || n == 0) return fail(GCG_ERR_INVALID, "gcg_mlp_train: bad argument");
    if (p->batch == 0 || p->batch % TRAIN_T) return fail(GCG_ERR_INVALID, "gcg_mlp_train: batch must be a multiple of 128");
    if (n >= 0xFFFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "gcg_mlp_train: at most 2^32-1 samples");
    cudaStream_t s = 0;
    GCG_TRY(set_train_smem());
    tbuf<float> xs, ts, part;
    tbuf<uint32_t> idx;
    tbuf<double> acc;
    const float *xd, *td;
    GCG_TRY(stage_in(x, (size_t)n * NIN, xs, &xd, s));
    GCG_TRY(stage_in(t, (size_t)n, ts, &td, s));
    const int grid = train_grid(p->batch);
    GCG_TRY(part.alloc((size_t)grid * (NP + 1), s));
    GCG_TRY(idx.alloc(n, s));
    GCG_TRY(acc.alloc(std::max<uint32_t>(p->epochs, 1), s));
    GCG_CUDA(cudaMemsetAsync(acc.get(), 0, (size_t)std::max<uint32_t>(p->epochs, 1) * 8, s));
    std::vector<uint32_t> order(n);
    uint32_t *h_order = nullptr; /* pinned: the upload of one epoch's order overlaps the previous epoch */
    GCG_CUDA(host_alloc((void **)&h_order, (size_t)n * 4));
    uint64_t rs = p->seed * 0x2545F4914F6CDD1Dull + 7;
    for (uint32_t ep = 0; ep < p->epochs; ++ep) {
        for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
        for (uint64_t i = n - 1; i > 0; --i) { /* Fisher-Yates */
            const uint64_t j = splitmix(rs) % (i + 1);
            std::swap(order[i], order[j]);
        }
        cudaStreamSynchronize(s); /* the previous epoch no longer reads the order */
        memcpy(h_order, order.data(), (size_t)n * 4);
        cudaError_t e = cudaMemcpyAsync(idx.get(), h_order, (size_t)n * 4, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            host_free(h_order);
            return fail(GCG_ERR_CUDA, std::string("gcg_mlp_train: ") + cudaGetErrorString(e));
        }
        for (uint64_t b0 = 0; b0 < n; b0 += p->batch) {
            const uint64_t cnt = std::min<uint64_t>(p->batch, n - b0);
            TrainArgs a;
            memset(&a, 0, sizeof(a));
            a.x = xd;
            a.t = td;
            a.idx = idx.get();
            a.base = b0;
            a.count = cnt;
            a.wb = m->wb.get();
            a.norm = m->norm.get();
            a.dscale = (float)(2.0 / (double)cnt);
            a.part = part.get();
            const int gb = train_grid(cnt);
            k_mlp_fwd_bwd<false><<<gb, TRAIN_T, TRAIN_SMEM, s>>>(a);
            ++m->step;
            AdamArgs d;
            memset(&d, 0, sizeof(d));
            d.part = part.get();
            d.nblocks = (uint32_t)gb;
            d.w = m->w.get();
            d.wb = m->wb.get();
            d.m = m->m.get();
            d.v = m->v.get();
            d.lr = p->lr;
            d.beta1 = p->beta1;
            d.beta2 = p->beta2;
            d.eps = p->eps;
            d.bc1 = (float)(1.0 - pow((double)p->beta1, (double)m->step));
            d.bc2 = (float)(1.0 - pow((double)p->beta2, (double)m->step));
            d.apply = 1;
            d.loss_acc = acc.get() + ep;
            k_mlp_adam<<<(NP + 1 + 255) / 256, 256, 0, s>>>(d);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            host_free(h_order);
            return fail(GCG_ERR_CUDA, std::string("gcg_mlp_train: launch: ") + cudaGetErrorString(e));
        }
    }
    cudaStreamSynchronize(s);
    host_free(h_order);
    GCG_TRY(mlp_prepare(m, s));
    std::vector<double> hl(std::max<uint32_t>(p->epochs, 1));
    GCG_CUDA(cudaMemcpyAsync(hl.data(), acc.get(), hl.size() * 8, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (epoch_loss)
        for (uint32_t ep = 0; ep < p->epochs; ++ep) epoch_loss[ep] = (float)(hl[ep] / (double)n);
    return GCG_OK;
}

int gcg_warm_start_rank(gcg_graph *g, const gcg_mlp *m, double teleport, double damping, float *init_rank,
                        double *device_ms) {
    if (!g || !m || !init_rank) return fail(GCG_ERR_INVALID, "gcg_warm_start_rank: null argument");
    if (!(teleport > 0.0)) return fail(GCG_ERR_INVALID, "gcg_warm_start_rank: teleport must be > 0");
    if (!(damping >= 0.0 && damping < 1.0)) return fail(GCG_ERR_INVALID, "gcg_warm_start_rank: damping must be in [0, 1)");
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    GCG_TRY(ensure_chunk_plan(g)); /* shared with PageRank; built once per graph */
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    int rc = GCG_OK;
    {
        const ChunkPlan &pl = *g->cplan;
        const int sms = num_sms();
        tbuf<Agg3> agg;
        tbuf<float> stage;
        tbuf<double2> pmass;
        tbuf<uint32_t> pzd;
        tbuf<double> alpha;
        tbuf<uint4> xpk;
        tbuf<int> ierr;
        float *dst = init_rank;
        const bool dev = is_device_ptr(init_rank);
        const uint64_t tiles = ((uint64_t)pl.nnz + TC_ROWS - 1) / TC_ROWS;
        /* at most TC_CTAS_PER_SM CTAs of 64 tensor-memory columns per SM: well inside its 512 */
        const unsigned ib = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, sms * (uint64_t)TC_CTAS_PER_SM));
        const unsigned zb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)pl.nzero + 255) / 256, sms * 4ull));
        rc = warm_aggregates(g, agg, s);
        if (rc == GCG_OK && !dev) {
            rc = stage.alloc(nv, s);
            dst = stage.get();
        }
        if (rc == GCG_OK && (rc = pmass.alloc(ib, s)) == GCG_OK && (rc = pzd.alloc(zb, s)) == GCG_OK &&
            (rc = alpha.alloc(1, s)) == GCG_OK && (rc = xpk.alloc(std::max<uint32_t>(pl.nnz, 1), s)) == GCG_OK &&
            (rc = ierr.alloc(1, s)) == GCG_OK && (rc = (cudaMemsetAsync(ierr.get(), 0, sizeof(int), s) == cudaSuccess
                                                            ? GCG_OK
                                                            : fail(GCG_ERR_CUDA, "gcg_warm_start_rank: memset"))) == GCG_OK) {
            const unsigned xb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)pl.nnz + 255) / 256, sms * 8ull));
            k_warm_xfeat<<<xb, 256, 0, s>>>(pl.nz_rows.get(), pl.od_nz.get(), pl.nnz, g->indeg.get(), agg.get(),
                                            g->vbits, m->norm.get(), xpk.get());
            InferArgs a;
            a.nz_rows = pl.nz_rows.get();
            a.od_nz = pl.od_nz.get();
            a.xpk = xpk.get();
            a.nnz = pl.nnz;
            a.wb = m->wb.get();
            a.teleport = (float)teleport;
            a.out = dst;
            a.part_mass = pmass.get();
            a.err = ierr.get();
            if (pl.nnz) k_warm_infer<<<ib, TC_ROWS, 0, s>>>(a);
            else cudaMemsetAsync(pmass.get(), 0, sizeof(double2), s);
            k_warm_zero<<<zb, 256, 0, s>>>(pl.zero_rows.get(), pl.nzero, g->outdeg.get(), (float)teleport, dst,
                                           pzd.get());
            k_warm_alpha<<<1, 32, 0, s>>>(pmass.get(), ib, pzd.get(), zb, nv, pl.nzero, teleport, damping,
                                          alpha.get());
            const unsigned sb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)pl.nnz + 255) / 256, sms * 8ull));
            k_warm_scale<<<sb, 256, 0, s>>>(pl.nz_rows.get(), pl.nnz, alpha.get(), dst);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(GCG_ERR_CUDA, std::string("gcg_warm_start_rank: ") + cudaGetErrorString(e));
        }
        cudaEventRecord(ev1, s);
        if (rc == GCG_OK && !dev) rc = copy_out(init_rank, dst, (size_t)nv * 4, s);
        int herr = 0;
        if (rc == GCG_OK && (cudaMemcpyAsync(&herr, ierr.get(), sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                             cudaStreamSynchronize(s) != cudaSuccess))
            rc = fail(GCG_ERR_CUDA, "gcg_warm_start_rank: readback");
        if (rc == GCG_OK && herr) rc = fail(GCG_ERR_TIMEOUT, "gcg_warm_start_rank: a tensor-core wait ran out");
    }
    cudaStreamSynchronize(s);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (device_ms) *device_ms = ms;
    return rc;
}

}  // extern "C"
