/*
 * Merge-path tiling of an in-edge CSR.
 *
 * The work of a pull sweep is the merge of two sorted lists: the row ends
 * (rowptr[1..V]) and the edge indices (0..E-1). Cutting that merge into tiles of
 * MP_TILE items gives every CTA the same number of rows + edges whatever the
 * degree skew (R-MAT hubs with 10^5 in-edges and long runs of empty rows alike).
 * Tile t covers rows [tile_row[t], tile_row[t+1]) that END in it and edges
 * [tile_edge[t], tile_edge[t+1]).
 *
 * A row whose edges began in an earlier tile (rowptr[r] < tile_edge[t]) is a
 * "head-split" row: its in-tile partial goes to head_part[t] and the row is
 * finished by a fix-up pass that adds the tail partials of the earlier tiles in
 * tile order, so every sum is computed in one fixed order (deterministic).
 */
#ifndef GCG_MERGEPATH_CUH
#define GCG_MERGEPATH_CUH

#include "gcg_internal.cuh"

namespace gcg {

/* Split point of diagonal `diag` in the merge of row ends a[0..na) with the
 * edge indices 0..nb-1 (a row end is taken before edge j when a[i] <= j). */
__device__ __forceinline__ uint32_t mp_search(const uint32_t *a, uint32_t na, uint32_t nb, uint32_t diag) {
    uint32_t lo = diag > nb ? diag - nb : 0u;
    uint32_t hi = diag < na ? diag : na;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] + mid + 1u <= diag) lo = mid + 1u; /* a[mid] <= diag - mid - 1 */
        else hi = mid;
    }
    return lo;
}

/* Same search over the global row pointers (a[i] = rowptr[i+1]), 64-bit diagonals. */
__device__ __forceinline__ uint32_t mp_search_global(const uint32_t *rowptr, uint32_t nv, uint64_t ne, uint64_t diag) {
    uint64_t lo = diag > ne ? diag - ne : 0ull;
    uint64_t hi = diag < nv ? diag : (uint64_t)nv;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if ((uint64_t)rowptr[mid + 1] + mid + 1ull <= diag) lo = mid + 1ull;
        else hi = mid;
    }
    return (uint32_t)lo;
}

/* Segmented scan element: f = "a row ended in this thread", v = running partial. */
struct SegVal {
    int f;
    float v;
};

/* Block-wide segmented scan over MP_THREADS threads. Returns the exclusive
 * prefix value for this thread (the carry into its first finished row) and
 * writes the block's inclusive total value to *total (all threads). */
__device__ __forceinline__ float seg_scan_excl(SegVal x, SegVal *s_warp, float *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    SegVal inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int fu = __shfl_up_sync(0xFFFFFFFFu, inc.f, o);
        float vu = __shfl_up_sync(0xFFFFFFFFu, inc.v, o);
        if (lane >= o) {
            if (!inc.f) inc.v = vu + inc.v;
            inc.f |= fu;
        }
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        SegVal w = (lane < MP_THREADS / 32) ? s_warp[lane] : SegVal{0, 0.0f};
#pragma unroll
        for (int o = 1; o < MP_THREADS / 32; o <<= 1) {
            int fu = __shfl_up_sync(0xFFFFFFFFu, w.f, o);
            float vu = __shfl_up_sync(0xFFFFFFFFu, w.v, o);
            if (lane >= o) {
                if (!w.f) w.v = vu + w.v;
                w.f |= fu;
            }
        }
        if (lane < MP_THREADS / 32) s_warp[lane] = w; /* inclusive over warps 0..lane */
    }
    __syncthreads();
    /* prefix of all earlier warps */
    SegVal wp = warp ? s_warp[warp - 1] : SegVal{0, 0.0f};
    /* inclusive of the previous lane in this warp */
    int fp = __shfl_up_sync(0xFFFFFFFFu, inc.f, 1);
    float vp = __shfl_up_sync(0xFFFFFFFFu, inc.v, 1);
    float excl;
    if (lane == 0) excl = wp.v;
    else excl = fp ? vp : wp.v + vp;
    *total = s_warp[MP_THREADS / 32 - 1].v;
    return excl;
}

}  // namespace gcg

#endif
