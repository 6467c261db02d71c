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
 *   k_warm_vstat   per vertex: {log(1+indeg), indeg} packed in 8 bytes
 *   k_warm_agg     per vertex with in-edges, 8 lanes per vertex: mean and max of
 *                  log(1+indeg(u)) over in-neighbours u and log(1 + sum indeg(u))
 *                  (one 8-byte gather per edge, FP64 sum, integer max and sum)
 *   k_warm_infer   fused features + network on tensor cores (mma.sync m16n8k16,
 *                  BF16 operands, FP32 accumulation): a warp runs 16 vertices,
 *                  layer 1 as 8 MMAs (K = 8 features padded to 16), layer 2 as 32
 *                  MMAs with the layer-1 accumulators re-packed in registers as
 *                  the A operand, layer 3 and exp on the FP32 pipes
 *   k_mlp_fwd_bwd  training: one sample per thread on the FP32 pipes (forward,
 *                  backward), then per-block weight gradients as small block
 *                  GEMMs over shared-memory activation tiles, one partial slot
 *                  per block (no atomics: the sum order is fixed)
 *   k_mlp_adam     fixed-order sum of the block partials, Adam on the FP32 master
 *                  weights, the BF16-rounded copy and the MMA operand fragments
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

namespace gcg {
namespace {

constexpr int NIN = GCG_MLP_IN;
constexpr int NH = GCG_MLP_HIDDEN;
constexpr int NP = GCG_MLP_NPARAMS;
/* offsets in the flat parameter vector */
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH;
static_assert(OB3 + 1 == NP, "parameter layout");
constexpr int NFRAG1 = 8 * 32;      /* layer-1 B fragments: 8 n-tiles x 32 lanes, one b32 each */
constexpr int NFRAG2 = 4 * 8 * 64;  /* layer-2 B fragments: 4 k-steps x 8 n-tiles x 32 lanes x 2 b32 */
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

__global__ void k_warm_vstat(const uint32_t *__restrict__ indeg, uint32_t nv, uint2 *__restrict__ vstat) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t d = indeg[v];
        const float L = (float)log1p((double)d);
        vstat[v] = make_uint2(__float_as_uint(L), d);
    }
}

/* agg[v] = {mean L(u), log(1 + max indeg(u)), log(1 + sum indeg(u))} over in-neighbours u */
__global__ void __launch_bounds__(256) k_warm_agg(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col,
                                                  const uint2 *__restrict__ vstat, uint32_t nv,
                                                  float4 *__restrict__ agg) {
    const uint32_t sub = threadIdx.x & 7u;
    const uint32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const uint32_t ngrp = (gridDim.x * blockDim.x) >> 3;
    /* every octet of a warp runs the same number of iterations (the shuffles are octet-local) */
    for (uint32_t base = grp - (grp & 3u); base < nv; base += ngrp) {
        const uint32_t v = base + (grp & 3u);
        double s = 0.0;
        uint32_t mx = 0;
        unsigned long long tot = 0;
        uint32_t b = 0, e = 0;
        if (v < nv) {
            b = rowptr[v];
            e = rowptr[v + 1];
        }
        for (uint32_t i = b + sub; i < e; i += 8u) {
            const uint2 x = vstat[col[i]];
            s += (double)__uint_as_float(x.x);
            mx = max(mx, x.y);
            tot += x.y;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
            mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
            tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
        }
        if (sub == 0 && v < nv) {
            const uint32_t d = e - b;
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if (d) {
                r.x = (float)(s / (double)d);
                r.y = (float)log1p((double)mx);
                r.z = (float)log1p((double)tot);
            }
            agg[v] = r;
        }
    }
}

/* the 8 raw features of vertex v */
__device__ __forceinline__ void raw_features(uint32_t v, uint32_t din, uint32_t dout, float4 ag, uint32_t vbits,
                                             float (&f)[NIN]) {
    f[0] = (float)log1p((double)din);
    f[1] = (float)log1p((double)dout);
    f[2] = ag.x;
    f[3] = ag.y;
    f[4] = ag.z;
    f[5] = dout ? (float)(1.0 / (double)dout) : 0.0f;
    f[6] = vbits >= 1 ? (float)((v >> (vbits - 1)) & 1u) : 0.0f;
    f[7] = vbits >= 2 ? (float)((v >> (vbits - 2)) & 1u) : 0.0f;
}

__global__ void k_warm_features(const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ outdeg,
                                const float4 *__restrict__ agg, uint32_t nv, uint32_t vbits, float *__restrict__ out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        float f[NIN];
        raw_features(v, indeg[v], outdeg[v], agg[v], vbits, f);
#pragma unroll
        for (int i = 0; i < NIN; ++i) out[(size_t)v * NIN + i] = f[i];
    }
}

/* ---- inference on tensor cores ------------------------------------------ */

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    return bf16_bits(lo) | (bf16_bits(hi) << 16);
}

/* D += A (16x16, row) * B (16x8, col), BF16 operands, FP32 accumulation */
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct InferArgs {
    const uint32_t *indeg, *outdeg;
    const float4 *agg;
    uint32_t nv, vbits;
    const uint32_t *frag1, *frag2; /* B operand fragments, lane-major */
    const float *wb;               /* rounded weights (biases FP32) */
    const float *norm;             /* mean[8], inv_std[8] */
    float teleport;
    float *out;
    double2 *part_mass;            /* per block: sum of the predicted ranks, of those without out-edges */
    ulonglong2 *part_count;        /* per block: vertices without in-edges, of those also without out-edges */
};

constexpr int INFER_THREADS = 256;

/* one warp = 16 vertices per step; lane (g = lane/4, t = lane%4) holds rows g and
 * g+8 of every accumulator tile (the m16n8 C layout), which is also the A layout
 * of the next layer once two adjacent n-tiles are packed to BF16 pairs */
__global__ void __launch_bounds__(INFER_THREADS) k_warm_infer(InferArgs a) {
    __shared__ float s_x[INFER_THREADS / 32][16][NIN + 1];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t g = lane >> 2, t = lane & 3u;
    uint32_t B1[8], B2[4][8][2];
    float bias1[8][2], bias2[8][2], w3[8][2];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        B1[nt] = a.frag1[nt * 32 + lane];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int c = nt * 8 + 2 * (int)t + q;
            bias1[nt][q] = a.wb[OB1 + c];
            bias2[nt][q] = a.wb[OB2 + c];
            w3[nt][q] = a.wb[OW3 + c];
        }
    }
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const uint2 f = ((const uint2 *)a.frag2)[(ks * 8 + nt) * 32 + lane];
            B2[ks][nt][0] = f.x;
            B2[ks][nt][1] = f.y;
        }
    const float b3 = a.wb[OB3];
    float mean[NIN], istd[NIN];
#pragma unroll
    for (int i = 0; i < NIN; ++i) {
        mean[i] = a.norm[i];
        istd[i] = a.norm[NIN + i];
    }
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t ntiles = (a.nv + 15u) >> 4;
    double msum = 0.0, mdang = 0.0;
    unsigned long long cz = 0, czd = 0;
    for (uint32_t tile = gwarp; tile < ntiles; tile += nwarps) {
        const uint32_t v0 = tile << 4;
        uint32_t din = 0, dout = 0;
        if (lane < 16) {
            const uint32_t v = v0 + lane;
            float f[NIN];
            if (v < a.nv) {
                din = a.indeg[v];
                dout = a.outdeg[v];
                raw_features(v, din, dout, a.agg[v], a.vbits, f);
            } else {
#pragma unroll
                for (int i = 0; i < NIN; ++i) f[i] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < NIN; ++i) s_x[warp][lane][i] = bf16r((f[i] - mean[i]) * istd[i]);
        }
        const uint32_t din_g = __shfl_sync(FULL, din, g), din_g8 = __shfl_sync(FULL, din, g + 8);
        const uint32_t dout_g = __shfl_sync(FULL, dout, g), dout_g8 = __shfl_sync(FULL, dout, g + 8);
        if (__ballot_sync(FULL, din != 0) == 0) { /* no vertex of the tile has in-edges */
            if (t == 0) {
                if (v0 + g < a.nv) {
                    a.out[v0 + g] = a.teleport;
                    ++cz;
                    czd += dout_g == 0;
                }
                if (v0 + g + 8 < a.nv) {
                    a.out[v0 + g + 8] = a.teleport;
                    ++cz;
                    czd += dout_g8 == 0;
                }
            }
            __syncwarp();
            continue;
        }
        __syncwarp();
        const uint32_t x0 = pack_bf16(s_x[warp][g][2 * t], s_x[warp][g][2 * t + 1]);
        const uint32_t x1 = pack_bf16(s_x[warp][g + 8][2 * t], s_x[warp][g + 8][2 * t + 1]);
        /* layer 1 -> A operand of layer 2 */
        uint32_t A2[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16(c, x0, x1, 0u, 0u, B1[nt], 0u);
            const float h0 = bf16r(fmaxf(c[0] + bias1[nt][0], 0.0f));
            const float h1 = bf16r(fmaxf(c[1] + bias1[nt][1], 0.0f));
            const float h2 = bf16r(fmaxf(c[2] + bias1[nt][0], 0.0f));
            const float h3 = bf16r(fmaxf(c[3] + bias1[nt][1], 0.0f));
            A2[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16(h0, h1);
            A2[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(h2, h3);
        }
        /* layer 2, then layer 3 on the FP32 pipes */
        float yg = 0.0f, yg8 = 0.0f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) mma_bf16(d, A2[ks][0], A2[ks][1], A2[ks][2], A2[ks][3], B2[ks][nt][0], B2[ks][nt][1]);
            yg = fmaf(fmaxf(d[0] + bias2[nt][0], 0.0f), w3[nt][0], yg);
            yg = fmaf(fmaxf(d[1] + bias2[nt][1], 0.0f), w3[nt][1], yg);
            yg8 = fmaf(fmaxf(d[2] + bias2[nt][0], 0.0f), w3[nt][0], yg8);
            yg8 = fmaf(fmaxf(d[3] + bias2[nt][1], 0.0f), w3[nt][1], yg8);
        }
        yg += __shfl_xor_sync(FULL, yg, 1);
        yg += __shfl_xor_sync(FULL, yg, 2);
        yg8 += __shfl_xor_sync(FULL, yg8, 1);
        yg8 += __shfl_xor_sync(FULL, yg8, 2);
        if (t == 0) {
            /* y is clamped so exp stays finite */
            const float y2[2] = {yg, yg8};
            const uint32_t di[2] = {din_g, din_g8}, dd[2] = {dout_g, dout_g8};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t v = v0 + g + 8 * q;
                if (v >= a.nv) continue;
                if (di[q]) {
                    const float r = a.teleport * expf(fminf(fmaxf(y2[q] + b3, -30.0f), 30.0f));
                    a.out[v] = r;
                    msum += (double)r;
                    if (dd[q] == 0) mdang += (double)r;
                } else {
                    a.out[v] = a.teleport;
                    ++cz;
                    czd += dd[q] == 0;
                }
            }
        }
        __syncwarp();
    }
    /* block partials of the mass terms, reduced in a fixed order */
    __shared__ double s_m[INFER_THREADS / 32][2];
    __shared__ unsigned long long s_c[INFER_THREADS / 32][2];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        msum += __shfl_xor_sync(FULL, msum, o);
        mdang += __shfl_xor_sync(FULL, mdang, o);
        cz += __shfl_xor_sync(FULL, cz, o);
        czd += __shfl_xor_sync(FULL, czd, o);
    }
    if (lane == 0) {
        s_m[warp][0] = msum;
        s_m[warp][1] = mdang;
        s_c[warp][0] = cz;
        s_c[warp][1] = czd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 m = make_double2(0.0, 0.0);
        ulonglong2 c = make_ulonglong2(0, 0);
        for (int w = 0; w < INFER_THREADS / 32; ++w) {
            m.x += s_m[w][0];
            m.y += s_m[w][1];
            c.x += s_c[w][0];
            c.y += s_c[w][1];
        }
        a.part_mass[blockIdx.x] = m;
        a.part_count[blockIdx.x] = c;
    }
}

/* Mass-stationary scale of the predicted ranks: alpha such that one Jacobi sweep
 * keeps the total rank. With Z = vertices without in-edges (rank = teleport
 * exactly), D = vertices without out-edges, M = sum of the predictions outside Z
 * and M_D = the part of M on D, the sweep's total is teleport*n +
 * damping*(total - total on D), which equals the total when
 *   alpha = teleport*(n - (1-damping)|Z| - damping|Z & D|) / ((1-damping)M + damping M_D). */
__global__ void k_warm_alpha(const double2 *__restrict__ pm, const ulonglong2 *__restrict__ pc, uint32_t nblocks,
                             uint32_t nv, double teleport, double damping, double *__restrict__ alpha) {
    const uint32_t lane = threadIdx.x;
    double M = 0.0, MD = 0.0;
    unsigned long long z = 0, zd = 0;
    for (uint32_t b = lane; b < nblocks; b += 32u) {
        M += pm[b].x;
        MD += pm[b].y;
        z += pc[b].x;
        zd += pc[b].y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        M += __shfl_xor_sync(0xFFFFFFFFu, M, o);
        MD += __shfl_xor_sync(0xFFFFFFFFu, MD, o);
        z += __shfl_xor_sync(0xFFFFFFFFu, z, o);
        zd += __shfl_xor_sync(0xFFFFFFFFu, zd, o);
    }
    if (lane == 0) {
        const double den = (1.0 - damping) * M + damping * MD;
        const double num = teleport * ((double)nv - (1.0 - damping) * (double)z - damping * (double)zd);
        *alpha = (den > 0.0 && num > 0.0) ? num / den : 1.0;
    }
}

__global__ void k_warm_scale(const uint32_t *__restrict__ indeg, uint32_t nv, const double *__restrict__ alpha,
                             float *__restrict__ out) {
    const double al = *alpha;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        if (indeg[v]) out[v] = (float)((double)out[v] * al);
}

/* B operand fragments of layers 1 and 2 from the rounded weights */
__global__ void k_mlp_pack(const float *__restrict__ wb, uint32_t *__restrict__ frag1, uint32_t *__restrict__ frag2) {
    for (uint32_t i = threadIdx.x; i < (uint32_t)NFRAG1; i += blockDim.x) {
        const uint32_t nt = i >> 5, lane = i & 31u, g = lane >> 2, t = lane & 3u;
        const float *w = wb + OW1 + (nt * 8 + g) * NIN;
        frag1[i] = pack_bf16(w[2 * t], w[2 * t + 1]);
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)(NFRAG2 / 2); i += blockDim.x) {
        const uint32_t lane = i & 31u, nt = (i >> 5) & 7u, ks = i >> 8, g = lane >> 2, t = lane & 3u;
        const float *w = wb + OW2 + (nt * 8 + g) * NH + ks * 16;
        frag2[2 * i] = pack_bf16(w[2 * t], w[2 * t + 1]);
        frag2[2 * i + 1] = pack_bf16(w[8 + 2 * t], w[8 + 2 * t + 1]);
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
    gcg::dbuf<uint32_t> frag;           /* MMA B fragments: layer 1 then layer 2 */
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

/* rounded copy and MMA fragments from the master weights (stream-ordered) */
int mlp_prepare(gcg_mlp *m, cudaStream_t s) {
    k_mlp_round<<<(NP + 255) / 256, 256, 0, s>>>(m->w.get(), m->wb.get());
    k_mlp_pack<<<1, 256, 0, s>>>(m->wb.get(), m->frag.get(), m->frag.get() + NFRAG1);
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

/* per-vertex aggregates of the in-neighbourhood (features 2-4) */
int warm_aggregates(gcg_graph *g, tbuf<float4> &agg, cudaStream_t s) {
    const uint32_t nv = g->nv;
    tbuf<uint2> vstat;
    GCG_TRY(vstat.alloc(nv, s));
    GCG_TRY(agg.alloc(nv, s));
    const int sms = num_sms();
    const unsigned b1 = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, sms * 8ull));
    k_warm_vstat<<<b1, 256, 0, s>>>(g->indeg.get(), nv, vstat.get());
    const unsigned b2 = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 31) / 32, sms * 8ull));
    k_warm_agg<<<b2, 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), vstat.get(), nv, agg.get());
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
        (rc = m->norm.alloc(2 * NIN)) || (rc = m->frag.alloc(NFRAG1 + NFRAG2))) {
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
    tbuf<float4> agg;
    GCG_TRY(warm_aggregates(g, agg, s));
    tbuf<float> stage;
    float *dst = features;
    const bool dev = is_device_ptr(features);
    if (!dev) {
        GCG_TRY(stage.alloc((size_t)nv * NIN, s));
        dst = stage.get();
    }
    const unsigned b = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, num_sms() * 8ull));
    k_warm_features<<<b, 256, 0, s>>>(g->indeg.get(), g->outdeg.get(), agg.get(), nv, g->vbits, dst);
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
    GCG_CUDA(cudaMallocHost((void **)&h_order, (size_t)n * 4));
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
            cudaFreeHost(h_order);
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
            cudaFreeHost(h_order);
            return fail(GCG_ERR_CUDA, std::string("gcg_mlp_train: launch: ") + cudaGetErrorString(e));
        }
    }
    cudaStreamSynchronize(s);
    cudaFreeHost(h_order);
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
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    int rc = GCG_OK;
    {
        tbuf<float4> agg;
        tbuf<float> stage;
        tbuf<double2> pmass;
        tbuf<ulonglong2> pcount;
        tbuf<double> alpha;
        float *dst = init_rank;
        const bool dev = is_device_ptr(init_rank);
        rc = warm_aggregates(g, agg, s);
        if (rc == GCG_OK && !dev) {
            rc = stage.alloc(nv, s);
            dst = stage.get();
        }
        if (rc == GCG_OK) {
            InferArgs a;
            a.indeg = g->indeg.get();
            a.outdeg = g->outdeg.get();
            a.agg = agg.get();
            a.nv = nv;
            a.vbits = g->vbits;
            a.frag1 = m->frag.get();
            a.frag2 = m->frag.get() + NFRAG1;
            a.wb = m->wb.get();
            a.norm = m->norm.get();
            a.teleport = (float)teleport;
            a.out = dst;
            const uint64_t warps = ((uint64_t)nv + 15) / 16;
            const unsigned blocks = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>((warps + INFER_THREADS / 32 - 1) / (INFER_THREADS / 32), num_sms() * 2ull));
            if ((rc = pmass.alloc(blocks, s)) == GCG_OK && (rc = pcount.alloc(blocks, s)) == GCG_OK &&
                (rc = alpha.alloc(1, s)) == GCG_OK) {
                a.part_mass = pmass.get();
                a.part_count = pcount.get();
                k_warm_infer<<<blocks, INFER_THREADS, 0, s>>>(a);
                k_warm_alpha<<<1, 32, 0, s>>>(pmass.get(), pcount.get(), blocks, nv, teleport, damping, alpha.get());
                const unsigned sb = (unsigned)std::max<uint64_t>(
                    1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, num_sms() * 8ull));
                k_warm_scale<<<sb, 256, 0, s>>>(g->indeg.get(), nv, alpha.get(), dst);
            }
        }
        if (rc == GCG_OK) {
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(GCG_ERR_CUDA, std::string("gcg_warm_start_rank: ") + cudaGetErrorString(e));
        }
        cudaEventRecord(ev1, s);
        if (rc == GCG_OK && !dev) rc = copy_out(init_rank, dst, (size_t)nv * 4, s);
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
