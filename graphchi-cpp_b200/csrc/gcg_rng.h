/*
 * Counter-based synthetic graph generators shared by host C and CUDA device code.
 *
 * The reference ships no R-MAT generator (src/util/graphgenerators.cpp has chain
 * and grid graphs only), so the seeded inputs are defined here. Every edge i is a
 * pure function of (seed, i): host threads and device threads produce bit-identical
 * edge lists, in any order and at any parallelism.
 *
 * R-MAT (Chakrabarti, Zhan, Faloutsos 2004): for edge i and level l in [0, scale),
 * a 32-bit uniform u_{i,l} picks the quadrant: u < a -> (0,0), < a+b -> (0,1),
 * < a+b+c -> (1,0), else (1,1); the chosen (src bit, dst bit) is appended below the
 * bits of earlier levels (most significant first). Thresholds are integers
 * floor(p * 2^32) computed once on the host. u_{i,l} is the high (l even) or low
 * (l odd) half of SplitMix64(seed_key + (i * ceil(scale/2) + l/2 + 1) * golden).
 *
 * Erdos-Renyi G(n, M): edge i takes one SplitMix64 draw; src = hi32 * n >> 32,
 * dst = lo32 * n >> 32.
 */
#ifndef GCG_RNG_H
#define GCG_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define GCG_HD __host__ __device__ __forceinline__
#else
#define GCG_HD static inline
#endif

#define GCG_GOLDEN 0x9E3779B97F4A7C15ULL

GCG_HD uint64_t gcg_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* Seed key: decorrelates nearby user seeds. */
GCG_HD uint64_t gcg_seed_key(uint64_t seed) { return gcg_mix64(seed ^ 0x6A09E667F3BCC909ULL); }

typedef struct {
    uint64_t ta, tab, tabc; /* cumulative quadrant thresholds, scaled by 2^32 */
} gcg_rmat_thresholds;

GCG_HD void gcg_rmat_edge(uint64_t key, uint64_t i, uint32_t scale, gcg_rmat_thresholds t,
                          uint32_t *src, uint32_t *dst) {
    uint32_t s = 0, d = 0;
    uint64_t ndraw = (scale + 1) / 2;
    uint64_t w = 0;
    for (uint32_t l = 0; l < scale; ++l) {
        if ((l & 1u) == 0) w = gcg_mix64(key + (i * ndraw + (l >> 1) + 1) * GCG_GOLDEN);
        uint64_t u = (l & 1u) ? (w & 0xFFFFFFFFULL) : (w >> 32);
        uint32_t q = (u < t.ta) ? 0u : (u < t.tab) ? 1u : (u < t.tabc) ? 2u : 3u;
        s = (s << 1) | (q >> 1);
        d = (d << 1) | (q & 1u);
    }
    *src = s;
    *dst = d;
}

GCG_HD void gcg_er_edge(uint64_t key, uint64_t i, uint32_t n, uint32_t *src, uint32_t *dst) {
    uint64_t w = gcg_mix64(key + (i + 1) * GCG_GOLDEN);
    *src = (uint32_t)(((w >> 32) * (uint64_t)n) >> 32);
    *dst = (uint32_t)(((w & 0xFFFFFFFFULL) * (uint64_t)n) >> 32);
}

#endif
