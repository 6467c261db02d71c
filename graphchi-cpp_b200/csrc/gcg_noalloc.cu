/*
 * PageRank (Jacobi) over an in-edge CSR that the caller already holds in device
 * memory, without allocating anything.
 *
 * Who needs this: callers that cannot let a library call cudaMalloc/cudaFree —
 * for example a host framework whose own caching allocator owns the GPU's memory
 * (a foreign cudaMalloc fragments or exceeds its budget), or a latency-bound loop
 * that must not hit the device-wide synchronisation cudaFree can cause. They pass
 * the graph, the out-degrees and the output vector in device memory they own;
 * everything else this call needs lives in one fixed-size scratch array below.
 *
 * Scratch: a file-scope __device__ array sized for NOALLOC_MAX_VERTICES vertices
 * (two contribution buffers, one spare rank buffer, the residual partials and
 * the control words: about 12.6 MB). Every GPU that loads this library holds it
 * until the process exits. Host code cannot use the symbol's name as a device
 * address; its address is fetched once per device with cudaGetSymbolAddress,
 * which happens on the first call on that device — make that first call before
 * any stream capture. Every call shares the array and it keeps the last call's
 * contents: the control words are cleared at the start of each call, and two
 * calls that overlap on the GPU (different streams, or host threads) race.
 * Every call waits for its stream before it returns (it reads the sweep count
 * and, with a tolerance, the convergence flag on the host). The arrays must be
 * device memory of the current device (or managed memory).
 */
#include <mutex>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

constexpr uint32_t NA_MAXV = GCG_NOALLOC_MAX_VERTICES;
constexpr uint32_t NA_BLOCKS = 1024; /* sweep kernel grid (residual partials) */
constexpr int NA_THREADS = 256;

/* scratch layout (byte offsets; every part 256-byte aligned) */
constexpr size_t NA_C_OFF = 0;                                  /* float c[2][NA_MAXV] */
constexpr size_t NA_R_OFF = NA_C_OFF + 2ull * NA_MAXV * 4;       /* float r_spare[NA_MAXV] */
constexpr size_t NA_PART_OFF = NA_R_OFF + (size_t)NA_MAXV * 4;   /* double2 part[NA_BLOCKS] */
constexpr size_t NA_CTL_OFF = NA_PART_OFF + (size_t)NA_BLOCKS * 16; /* uint32 ticket, done, sweeps, pad */
constexpr size_t NA_RES_OFF = NA_CTL_OFF + 256;                  /* double last residual, u64 t0, u64 t1 */
constexpr size_t NA_BYTES = NA_RES_OFF + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NaArgs {
    const uint32_t *rowptr, *col, *outdeg;
    uint32_t nv;
    const float *c_old;
    float *c_new;
    const float *r_old;
    float *r_new;
    double2 *part;
    uint32_t *ticket;
    int *done, *sweeps;
    double *res;
    double *res_log; /* caller's residuals[] or NULL: written by the sweeps that run */
    unsigned long long *t_end;
    double teleport, damping, tol;
};

/* the GPU's global nanosecond timer */
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void k_na_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float init, const float *__restrict__ init_rank,
                          float *__restrict__ r, float *__restrict__ c, unsigned long long *t_start) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *t_start = globaltimer_ns();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const float x = init_rank ? init_rank[v] : init;
        r[v] = x;
        const uint32_t od = outdeg[v];
        c[v] = od ? __fdiv_rn(x, (float)od) : 0.0f;
    }
}

/* One sweep: a warp per row (lane-strided sum, fixed shuffle tree), apply, and a
 * fixed-order FP64 residual reduction by the last block to finish. */
__global__ void __launch_bounds__(NA_THREADS) k_na_sweep(NaArgs a, int sweep) {
    if (*(volatile const int *)a.done) return;
    __shared__ double2 s_red[NA_THREADS / 32];
    __shared__ int s_last;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    double dsum = 0.0, nsum = 0.0;
    for (uint32_t v = gw; v < a.nv; v += nw) {
        float s = 0.0f;
        for (uint32_t j = a.rowptr[v] + lane; j < a.rowptr[v + 1]; j += 32u) s += a.c_old[a.col[j]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
        if (lane == 0) {
            const float rn = (float)__dadd_rn(a.teleport, __dmul_rn(a.damping, (double)s));
            const float ro = a.r_old[v];
            a.r_new[v] = rn;
            const uint32_t od = a.outdeg[v];
            a.c_new[v] = od ? __fdiv_rn(rn, (float)od) : 0.0f;
            dsum += fabs((double)rn - (double)ro);
            nsum += fabs((double)rn);
        }
    }
    if (lane == 0) s_red[warp] = make_double2(dsum, nsum);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < NA_THREADS / 32; ++w) {
            t.x += s_red[w].x;
            t.y += s_red[w].y;
        }
        a.part[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    double x = 0.0, y = 0.0;
    for (uint32_t b = 0; b < gridDim.x; ++b) {
        const double2 p = __ldcg(a.part + b);
        x += p.x;
        y += p.y;
    }
    const double res = y > 0.0 ? x / y : 0.0;
    *a.res = res;
    if (a.res_log) a.res_log[sweep] = res;
    *a.sweeps = sweep + 1;
    *a.t_end = globaltimer_ns();
    if (a.tol > 0.0 && res <= a.tol) *a.done = 1;
    *a.ticket = 0u;
}

/* Device address of the scratch array, fetched once per device. */
std::mutex g_na_mutex;
unsigned char *g_na_ptr[64] = {nullptr};

int scratch_address(unsigned char **out) {
    int dev = 0;
    GCG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(GCG_ERR_UNSUPPORTED, "gcg_pagerank_csr_noalloc: device index >= 64");
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(GCG_ERR_CUDA, std::string("gcg_pagerank_csr_noalloc: cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e));
        g_na_ptr[dev] = (unsigned char *)p;
    }
    *out = g_na_ptr[dev];
    return GCG_OK;
}

/* device memory of device dev (or managed memory, reachable from every device) */
bool on_device(const void *p, int dev) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError(); /* clear: unregistered host pointer */
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace
}  // namespace gcg

using namespace gcg;

extern "C" int gcg_pagerank_csr_noalloc(const uint32_t *in_rowptr, const uint32_t *in_col, const uint32_t *outdeg,
                                        uint32_t num_vertices, const gcg_pr_params *params, float *out_rank,
                                        void *stream, gcg_pr_stats *stats) {
    if (!in_rowptr || !in_col || !outdeg || !params || !out_rank)
        return fail(GCG_ERR_INVALID, "gcg_pagerank_csr_noalloc: null argument");
    if (num_vertices == 0) return fail(GCG_ERR_INVALID, "gcg_pagerank_csr_noalloc: num_vertices must be > 0");
    if (num_vertices > NA_MAXV)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_pagerank_csr_noalloc: " + std::to_string(num_vertices) +
                                             " vertices exceed the fixed scratch limit of " +
                                             std::to_string(NA_MAXV) + " (GCG_NOALLOC_MAX_VERTICES)");
    if (params->mode != GCG_PR_JACOBI || params->source != GCG_NO_SOURCE)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_pagerank_csr_noalloc: only plain GCG_PR_JACOBI is available");
    if (params->max_sweeps < 0) return fail(GCG_ERR_INVALID, "gcg_pagerank_csr_noalloc: max_sweeps < 0");
    int dev = 0;
    GCG_CUDA(cudaGetDevice(&dev));
    if (!on_device(in_rowptr, dev) || !on_device(in_col, dev) || !on_device(outdeg, dev) || !on_device(out_rank, dev) ||
        (params->init_rank && !on_device(params->init_rank, dev)) ||
        (params->residuals && !on_device(params->residuals, dev)))
        return fail(GCG_ERR_INVALID,
                    "gcg_pagerank_csr_noalloc: every array must be device memory of the current device "
                    "(this entry point allocates nothing)");
    unsigned char *base = nullptr;
    GCG_TRY(scratch_address(&base));
    cudaStream_t s = (cudaStream_t)stream;

    float *c = (float *)(base + NA_C_OFF);
    float *r_spare = (float *)(base + NA_R_OFF);
    uint32_t *ctl = (uint32_t *)(base + NA_CTL_OFF);
    NaArgs a;
    a.rowptr = in_rowptr;
    a.col = in_col;
    a.outdeg = outdeg;
    a.nv = num_vertices;
    a.part = (double2 *)(base + NA_PART_OFF);
    a.ticket = ctl;
    a.done = (int *)(ctl + 1);
    a.sweeps = (int *)(ctl + 2);
    a.res = (double *)(base + NA_RES_OFF);
    a.res_log = params->residuals;
    unsigned long long *t_dev = (unsigned long long *)(base + NA_RES_OFF + 8); /* start, end */
    a.t_end = t_dev + 1;
    a.teleport = params->teleport;
    a.damping = params->damping;
    a.tol = params->tol;
    /* the array keeps the previous call's contents: clear the control words */
    GCG_CUDA(cudaMemsetAsync(base + NA_CTL_OFF, 0, 256 + 256, s));
    unsigned ib = (unsigned)std::min<uint64_t>(((uint64_t)num_vertices + 255) / 256, (uint64_t)num_sms() * 8);
    k_na_init<<<ib, 256, 0, s>>>(num_vertices, outdeg, params->init, params->init_rank, out_rank, c, t_dev);
    GCG_LAUNCH_CHECK();
    /* ranks ping-pong between the caller's output and the spare buffer */
    float *rb[2] = {out_rank, r_spare};
    const unsigned grid = (unsigned)std::min<uint64_t>(((uint64_t)num_vertices + 7) / 8, NA_BLOCKS);
    int launched = 0;
    int flags[2] = {0, 0};
    while (launched < params->max_sweeps) {
        const int n = std::min(4, params->max_sweeps - launched);
        for (int k = 0; k < n; ++k) {
            const int sw = launched + k;
            a.c_old = c + (size_t)(sw & 1) * NA_MAXV;
            a.c_new = c + (size_t)((sw + 1) & 1) * NA_MAXV;
            a.r_old = rb[sw & 1];
            a.r_new = rb[(sw + 1) & 1];
            k_na_sweep<<<grid, NA_THREADS, 0, s>>>(a, sw);
        }
        GCG_LAUNCH_CHECK();
        launched += n;
        if (params->tol > 0.0) {
            GCG_CUDA(cudaMemcpyAsync(flags, ctl + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            if (flags[0]) break;
        }
    }
    GCG_CUDA(cudaMemcpyAsync(flags, ctl + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    double res = 0.0;
    unsigned long long t_ns[2] = {0, 0};
    GCG_CUDA(cudaMemcpyAsync(&res, a.res, sizeof(double), cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaMemcpyAsync(t_ns, t_dev, sizeof(t_ns), cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    const int sweeps = flags[1];
    if (sweeps & 1) { /* the result sits in the spare buffer */
        GCG_CUDA(cudaMemcpyAsync(out_rank, r_spare, (size_t)num_vertices * 4, cudaMemcpyDeviceToDevice, s));
        GCG_CUDA(cudaStreamSynchronize(s));
    }
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = flags[0];
        stats->residual = res;
        /* GPU global timer: start of the initial-vector kernel to the end of the last sweep that ran */
        stats->device_ms = (sweeps > 0 && t_ns[1] > t_ns[0]) ? (double)(t_ns[1] - t_ns[0]) * 1e-6 : 0.0;
        stats->sweep_kernel_ms = 0.0;
        stats->timed_sweeps = 0;
        stats->kernel_launches = 1 + launched;
        stats->levels = 0;
    }
    return GCG_OK;
}
