/*
 * graphchi_gpu functional plug-in on the device: runs a user's gather-apply-
 * scatter kernel (functional_kernel<VT, ET>, functional_api.hpp:54-75) on the
 * graph the shim shards into HBM. Compile the file that includes this header
 * with nvcc (-gencode arch=compute_100a,code=sm_100a) and link libgcgpu; mark
 * the kernel's methods GCG_HD.
 *
 * Semantics of run_functional_unweighted_synchronous (functional_bulksync.hpp:51-169):
 *   iteration 0: v = initial_value(ctx, v)
 *   iteration i >= 1: sum = reset(); for every in-edge u -> v,
 *     sum = plus(sum, op_neighborval(ctx_i, v, u, value_to_neighbor(ctx_{i-1}, u, v, value_{i-1}(u))));
 *     v = compute_vertexvalue(ctx_i, v, sum)
 * The edge value u writes in iteration i-1 is computed where v gathers it, from
 * u's previous value, so no per-edge storage is needed; values are double
 * buffered (bulk-synchronous). One warp per vertex: lanes evaluate scatter and
 * gather for 32 in-edges at a time, lane 0 folds them with plus in ascending
 * source order (the reference's order is lock-striped and varies; this one is
 * fixed, so runs are deterministic). Writes <file>.<sizeof(VT)>B.vout.
 *
 * run_functional_unweighted_semisynchronous runs the same bulk-synchronous
 * schedule: the reference's semi-synchronous mode reads values of the running
 * iteration in an order that depends on its threads; results agree to the
 * kernel's convergence, not bit for bit.
 */
#ifndef GRAPHCHI_GPU_FUNCTIONAL_CUH
#define GRAPHCHI_GPU_FUNCTIONAL_CUH

#include <cuda_runtime.h>

#include "graphchi_gpu.hpp"

namespace graphchi {
namespace functional_detail {

constexpr int WARPS = 8;

template <typename KERNEL>
__global__ void k_initial(KERNEL kern, graphchi_context ctx, const uint32_t *indeg, const uint32_t *outdeg,
                          uint32_t nv, typename KERNEL::VertexDataType *val) {
    KERNEL k = kern;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        vertex_info vi{v, (int)indeg[v], (int)outdeg[v]};
        graphchi_context c = ctx;
        val[v] = k.initial_value(c, vi);
    }
}

template <typename KERNEL>
__global__ void __launch_bounds__(WARPS * 32) k_step(KERNEL kern, graphchi_context ctx, graphchi_context prev,
                                                     gcg_graph_device_view g,
                                                     const typename KERNEL::VertexDataType *old_val,
                                                     typename KERNEL::VertexDataType *new_val) {
    typedef typename KERNEL::VertexDataType VT;
    typedef typename KERNEL::EdgeDataType ET;
    __shared__ ET s_val[WARPS][32];
    KERNEL k = kern;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < g.num_vertices; v += nwarps) {
        vertex_info vi{v, (int)g.indeg[v], (int)g.outdeg[v]};
        const uint32_t b = g.in_rowptr[v], e = g.in_rowptr[v + 1];
        VT sum = VT();
        if (lane == 0) sum = k.reset();
        for (uint32_t base = b; base < e; base += 32u) {
            const uint32_t i = base + lane;
            if (i < e) {
                const uint32_t u = g.in_col[i];
                vertex_info ui{u, (int)g.indeg[u], (int)g.outdeg[u]};
                graphchi_context cp = prev, cc = ctx;
                const ET ev = k.value_to_neighbor(cp, ui, v, old_val[u]);
                s_val[warp][lane] = k.op_neighborval(cc, vi, u, ev);
            }
            __syncwarp();
            if (lane == 0) {
                const uint32_t n = e - base < 32u ? e - base : 32u;
                for (uint32_t j = 0; j < n; ++j) sum = k.plus(sum, s_val[warp][j]);
            }
            __syncwarp();
        }
        if (lane == 0) {
            graphchi_context cc = ctx;
            new_val[v] = k.compute_vertexvalue(cc, vi, sum);
        }
    }
}

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw gcg_error(GCG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace functional_detail

template <typename KERNEL>
void run_functional_unweighted_synchronous(std::string filename, int niters, metrics &m) {
    using namespace functional_detail;
    typedef typename KERNEL::VertexDataType VT;
    typedef typename KERNEL::EdgeDataType ET;
    /* edges hold a pair of values in the reference's shards (PairContainer<ET>) */
    gpu_convert(filename, get_option_string("nshards", "auto"), 2 * sizeof(ET));
    gcg_graph *gr = gpu_graphs()[filename]->g;
    gcg_graph_device_view g;
    gcg_check(gcg_graph_get_device_view(gr, &g), "device view");
    cudaStream_t s = (cudaStream_t)g.stream;
    const uint32_t nv = g.num_vertices;
    VT *a = nullptr, *b = nullptr;
    cuda_check(cudaMalloc((void **)&a, sizeof(VT) * std::max<uint32_t>(nv, 1)), "cudaMalloc");
    if (cudaMalloc((void **)&b, sizeof(VT) * std::max<uint32_t>(nv, 1)) != cudaSuccess) {
        cudaFree(a);
        throw gcg_error(GCG_ERR_NOMEM, "cudaMalloc of the vertex values failed");
    }
    m.start_time("runtime");
    graphchi_context ctx;
    ctx.nvertices = nv;
    ctx.nedges = g.num_edges;
    ctx.num_iterations = niters;
    ctx.filename = nullptr; /* host memory: not handed to the device */
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned vb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + 255) / 256, sms * 8ull));
    const unsigned sb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv + WARPS - 1) / WARPS,
                                                                         sms * 16ull));
    KERNEL kern;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    if (niters > 0) {
        ctx.iteration = 0;
        k_initial<KERNEL><<<vb, 256, 0, s>>>(kern, ctx, g.indeg, g.outdeg, nv, a);
    }
    for (int it = 1; it < niters; ++it) {
        graphchi_context prev = ctx;
        ctx.iteration = it;
        k_step<KERNEL><<<sb, WARPS * 32, 0, s>>>(kern, ctx, prev, g, a, b);
        std::swap(a, b);
    }
    cudaEventRecord(e1, s);
    cudaError_t err = cudaStreamSynchronize(s);
    if (err == cudaSuccess) err = cudaGetLastError();
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<VT> host(nv);
    if (err == cudaSuccess) err = cudaMemcpy(host.data(), a, sizeof(VT) * nv, cudaMemcpyDeviceToHost);
    cudaFree(a);
    cudaFree(b);
    cuda_check(err, "functional kernel");
    m.add_time("device_functional", ms / 1000.0);
    gcg_check(gcg_write_vout(filename.c_str(), host.data(), nv, sizeof(VT)), "write vout");
    m.stop_time("runtime");
}

template <typename KERNEL>
void run_functional_unweighted_semisynchronous(std::string filename, int niters, metrics &m) {
    run_functional_unweighted_synchronous<KERNEL>(filename, niters, m);
}

}  // namespace graphchi

#endif
