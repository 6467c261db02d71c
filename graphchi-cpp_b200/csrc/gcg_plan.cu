/*
 * Merge-path tiling of the in-edge CSR (see gcg_mergepath.cuh), built once per
 * graph and used by the edge passes of connected components and triangle
 * counting.
 */
#include <algorithm>

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

}  // namespace

int ensure_plan(gcg_graph *g) {
    if (g->plan) return GCG_OK;
    PrPlan *p = new PrPlan();
    const uint64_t total = (uint64_t)g->nv + g->ne;
    p->ntiles = (uint32_t)((total + MP_TILE - 1) / MP_TILE);
    if (p->tile_row.alloc((size_t)p->ntiles + 1) || p->tile_edge.alloc((size_t)p->ntiles + 1)) {
        delete p;
        return GCG_ERR_NOMEM;
    }
    unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)p->ntiles + 256) / 256, 4096));
    k_plan<<<blocks, 256, 0, g->stream>>>(g->in_rowptr.get(), g->nv, g->ne, p->ntiles, p->tile_row.get(),
                                          p->tile_edge.get());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        delete p;
        return fail(GCG_ERR_CUDA, std::string("merge-path plan: ") + cudaGetErrorString(e));
    }
    g->plan = p;
    return GCG_OK;
}

}  // namespace gcg
