/*
 * Merge-path tiling of an in-edge CSR.
 *
 * The work of a pull sweep is the merge of two sorted lists: the row ends
 * (rowptr[1..V]) and the edge indices (0..E-1). Cutting that merge into tiles of
 * MP_TILE items gives every CTA the same number of rows + edges whatever the
 * degree skew (R-MAT hubs with 10^5 in-edges and long runs of empty rows alike).
 * Tile t covers rows [tile_row[t], tile_row[t+1]) that END in it and edges
 * [tile_edge[t], tile_edge[t+1]).
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

}  // namespace gcg

#endif
