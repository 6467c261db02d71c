/*
 * Exact vertex-API PageRank: the in-memory program of example_apps/pagerank.cpp
 * (:121-146) as the engine runs it with deterministic parallelism
 * (src/engine/graphchi_engine.hpp:396-454): one Gauss-Seidel sweep per iteration
 * in ascending vertex id order, each vertex reading the values its smaller-id
 * in-neighbours wrote in this sweep and its larger-id in-neighbours' values from
 * the previous sweep, summing them in ascending source order in float.
 *
 * Parallel form: vertex v depends on in-neighbours u < v only, so v's level
 * (1 + max level of those u, 0 if none) orders the sweep: every level is a set of
 * independent vertices. Within a sweep, levels run in order; each vertex sums
 * sequentially (bit-exact float order), reading new values below its id and old
 * values above it. Levels come from a monotone relaxation over the in-CSR and a
 * radix sort of (level, id); the per-level launches of one sweep are captured
 * once in a CUDA graph and replayed per sweep.
 *
 * The same schedule runs the edge-value program of the app (PagerankProgram,
 * example_apps/pagerank.cpp:73-113, taken when num_vertices * 4 >= membudget):
 * there the value on every out-edge of u is u's pagerank / outdeg in float,
 * initially (float)(1.0/outdeg), the vertex value is the pagerank itself, and
 * each iteration logs the sum of |pagerank - old| (pagerank.cpp:108).
 */
#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

/* Levels of the id-ordered dependency DAG (edges u -> v with u < v) by
 * topological rounds (Kahn): a vertex's level is 1 + the largest level of its
 * smaller-id in-neighbours, i.e. the round after its last such neighbour's. */

/* pending[v] = number of in-neighbours u < v (sources ascending: a binary search) */
__global__ void k_gs_pending(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                             uint32_t *__restrict__ pending) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t lo = rowptr[v], hi = rowptr[v + 1]; /* first position with col >= v */
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if (col[mid] < v) lo = mid + 1; else hi = mid;
        }
        pending[v] = lo - rowptr[v];
    }
}

/* keys (u << vbits) | v of the edges u -> v with u < v, compacted by a scan
 * over the per-vertex counts */
__global__ void k_gs_fwd_keys(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                              const uint32_t *__restrict__ pending, const uint32_t *__restrict__ pos, uint32_t vbits,
                              uint64_t *__restrict__ keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t b = rowptr[v], n = pending[v], o = pos[v];
        for (uint32_t j = 0; j < n; ++j) keys[o + j] = ((uint64_t)col[b + j] << vbits) | v;
    }
}

/* fwd_off[u] = first sorted key with source >= u (keys sorted by source) */
__global__ void k_gs_fwd_off(const uint64_t *__restrict__ keys, uint64_t n, uint32_t vbits, uint32_t nv,
                             uint32_t *__restrict__ off, uint32_t *__restrict__ dst) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        dst[i] = (uint32_t)(k & mask);
        const int64_t u = (int64_t)(k >> vbits);
        const int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> vbits);
        for (int64_t x = prev + 1; x <= u; ++x) off[x] = (uint32_t)i;
        if (i == n - 1)
            for (int64_t x = u + 1; x <= (int64_t)nv; ++x) off[x] = (uint32_t)n;
    }
}

/* round 0: the vertices without smaller-id in-neighbours */
__global__ void k_gs_roots(const uint32_t *__restrict__ pending, uint32_t nv, uint32_t *__restrict__ front,
                           uint32_t *__restrict__ count) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        if (pending[v] == 0) front[atomicAdd(count, 1u)] = v;
}

/* one round: a warp per vertex of the current frontier (level r) releases its
 * forward edges; a vertex whose last pending in-neighbour this is joins the next
 * frontier with level r + 1. Counts per round: cnt[r] = frontier size of round
 * r; rounds whose frontier is empty return at once (several are queued). */
__global__ void __launch_bounds__(256) k_gs_round(uint32_t r, const uint32_t *__restrict__ fwd_off,
                                                  const uint32_t *__restrict__ fwd_dst, uint32_t *pending,
                                                  uint32_t *level, const uint32_t *__restrict__ front_cur,
                                                  uint32_t *front_next, uint32_t *cnt) {
    const uint32_t n = *(volatile const uint32_t *)(cnt + r);
    if (n == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const uint32_t u = front_cur[i];
        for (uint32_t j = fwd_off[u] + lane; j < fwd_off[u + 1]; j += 32) {
            const uint32_t v = fwd_dst[j];
            if (atomicSub(pending + v, 1u) == 1u) {
                level[v] = r + 1;
                front_next[atomicAdd(cnt + r + 1, 1u)] = v;
            }
        }
    }
}

/* Vertex classes of a level, by in-degree: a thread sums a row of at most
 * GS_THREAD_MAX in-edges, a warp one of at most GS_WARP_MAX, a block a longer
 * one. Every class adds the in-edges one after another in ascending source
 * order (a float sum is not associative); the cooperating threads only load. */
/* R-MAT scale 22, per sweep: warp limit 1024: 31.8 ms, 512: 31.1, 256: 29.0, 128: 29.1
 * (scale 24: 88.6 ms for all four) */
constexpr uint32_t GS_THREAD_MAX = 32, GS_WARP_MAX = 256;
constexpr int GS_CLASSES = 4; /* segments per level: thread, warp, block, (unused) */

/* sort key: level, class, vertex id */
__global__ void k_level_keys(const uint32_t *__restrict__ level, const uint32_t *__restrict__ rowptr, uint32_t nv,
                             uint32_t vbits, uint64_t *keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t d = rowptr[v + 1] - rowptr[v];
        const uint64_t cls = d <= GS_THREAD_MAX ? 0u : d <= GS_WARP_MAX ? 1u : 2u;
        keys[v] = ((((uint64_t)level[v] << 2) | cls) << vbits) | v;
    }
}

/* order[i] = vertex of sorted key i; off[x] = first i whose segment
 * (level * GS_CLASSES + class) is >= x, for x in [0, nseg] */
__global__ void k_level_bounds(const uint64_t *__restrict__ keys, uint32_t nv, uint32_t vbits, uint32_t nseg,
                               uint32_t *__restrict__ off, uint32_t *__restrict__ order) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        order[i] = (uint32_t)(k & mask);
        int64_t l = (int64_t)(k >> vbits);
        int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> vbits);
        for (int64_t x = prev + 1; x <= l; ++x) off[x] = i;
        if (i == nv - 1)
            for (int64_t x = l + 1; x <= (int64_t)nseg; ++x) off[x] = nv;
    }
}


/* pagerank.cpp:124,137-139: pr starts at 0.15; iteration 0 sets 1/outc when outc > 0 */
__global__ void k_gs_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float reset, float *pr) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t oc = outdeg[v];
        pr[v] = oc > 0 ? __fdiv_rn(1.0f, (float)oc) : reset;
    }
}

/* pagerank.cpp:80-83 (edge-value program, iteration 0): out-edges hold
 * (float)(1.0 / outdeg) */
__global__ void k_gs_edge_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float *c) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t oc = outdeg[v];
        c[v] = oc > 0 ? __double2float_rn(__ddiv_rn(1.0, (double)oc)) : 0.0f;
    }
}

/* 4-byte asynchronous copy global -> shared (through L1), in commit groups */
__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
/* block class: steps of GS_STEP values, GS_DEPTH of them in flight (per sweep
 * at R-MAT scale 24, 10 sweeps: 1024 x 2 88.6 ms, 1024 x 3 90.1, 1024 x 4 90.7,
 * 2048 x 2 88.0, 2048 x 3 92.7, 512 x 2 116.1, 512 x 3 119.7, 256 x 3 108.2) */
constexpr uint32_t GS_STEP = 1024, GS_DEPTH = 2;

/* value of in-edge (u -> v): this sweep's for u < v (an earlier level, written
 * by an earlier launch), the previous sweep's otherwise */
__device__ __forceinline__ float gs_in_value(uint32_t u, uint32_t v, const float *__restrict__ pr_old,
                                             const float *__restrict__ pr_new) {
    return u < v ? __ldg(pr_new + u) : __ldg(pr_old + u);
}

/* The apply of one vertex. In-memory program (EDGE = false), pagerank.cpp:127-136:
 * pr = (float)((0.15 + 0.85 * (double)sum) / outc). Edge-value program (EDGE =
 * true), pagerank.cpp:89-111: pagerank = (float)(0.15 + 0.85 * (double)sum), the
 * out-edge value pagerank / outc in float. TRACK (always with EDGE): the vertex's
 * pagerank goes to val[v] and |pagerank - previous| (float) to delta[v], for
 * the progress log and the residual stop. Explicit round-to-nearest ops: no FMA
 * contraction, the same rounding as the reference's separate double multiply
 * and add. */
template <bool EDGE, bool TRACK>
__device__ __forceinline__ void gs_apply(uint32_t v, float sum, const uint32_t *__restrict__ outdeg, float *pr_new,
                                         float *val, float *delta, double reset, double damping) {
    const int outc = (int)outdeg[v];
    const double t = __dadd_rn(reset, __dmul_rn(damping, (double)sum));
    if (EDGE) pr_new[v] = outc > 0 ? __fdiv_rn(__double2float_rn(t), (float)outc) : 0.0f;
    else pr_new[v] = outc > 0 ? (float)__ddiv_rn(t, (double)outc) : (float)t;
    if (TRACK) {
        const float pagerank = __double2float_rn(t);
        delta[v] = fabsf(__fsub_rn(pagerank, val[v]));
        val[v] = pagerank;
    }
}

/* One level of a sweep: the level's vertices are independent. Blocks
 * [0, nb) take the block-class vertices (one each: the threads copy the
 * in-edge values of a GS_STEP-edge step into shared memory, GS_DEPTH steps in
 * flight, thread 0 adds the step in order); the next blocks take the
 * warp-class vertices (one per warp: 32 values per batch, lane 0 adds them in
 * order from shuffles, the next batch already loading); the rest take the
 * thread-class vertices (eight loads in flight, then eight adds in order).
 * Levels of sweeps queued after `done` was raised return at once. */
template <bool EDGE, bool TRACK>
__global__ void __launch_bounds__(256) k_gs_level(const uint32_t *__restrict__ order, uint32_t tb, uint32_t wb,
                                                  uint32_t bb, uint32_t be, const uint32_t *__restrict__ rowptr,
                                                  const uint32_t *__restrict__ col,
                                                  const uint32_t *__restrict__ outdeg,
                                                  const float *__restrict__ pr_old, float *pr_new, float *val,
                                                  float *delta, const int *done, double reset, double damping) {
    if (TRACK && *(volatile const int *)done) return;
    const uint32_t nb = be - bb, nwb = (bb - wb + 7) / 8;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (blockIdx.x < nb) { /* block class */
        /* GS_DEPTH steps of GS_STEP in-edge values in flight: every thread copies
         * GS_STEP / 256 values of a step into shared memory with cp.async (the
         * source columns read one step ahead), so the loads of the next step
         * overlap thread 0's in-order adds of the current one */
        constexpr uint32_t GQ = GS_STEP / 256;
        __shared__ __align__(16) float s_val[GS_DEPTH][GS_STEP];
        const uint32_t v = order[bb + blockIdx.x];
        const uint32_t jb = rowptr[v], je = rowptr[v + 1];
        const uint32_t nstep = (je - jb + GS_STEP - 1) / GS_STEP;
        float sum = 0.0f;
        /* this thread's copies for step b (source columns u), then one commit
         * group per step, empty past the row's end */
        auto issue = [&](uint32_t b, const uint32_t (&u)[GQ]) {
#pragma unroll
            for (uint32_t q = 0; q < GQ; ++q)
                if (b < nstep && jb + b * GS_STEP + q * 256 + tid < je)
                    cp_async4(&s_val[b % GS_DEPTH][q * 256 + tid], (u[q] < v ? pr_new : pr_old) + u[q]);
            cp_async_commit();
        };
        auto columns = [&](uint32_t b, uint32_t (&u)[GQ]) {
#pragma unroll
            for (uint32_t q = 0; q < GQ; ++q) {
                const uint32_t j = jb + b * GS_STEP + q * 256 + tid;
                u[q] = b < nstep && j < je ? __ldg(col + j) : 0u;
            }
        };
        uint32_t cn[GQ];
        for (uint32_t b = 0; b + 1 < GS_DEPTH; ++b) {
            columns(b, cn);
            issue(b, cn);
        }
        columns(GS_DEPTH - 1, cn);
        for (uint32_t b = 0; b < nstep; ++b) {
            cp_async_wait<GS_DEPTH - 2>(); /* this thread's values of step b have landed */
            __syncthreads();               /* everyone's; thread 0 is done with step b - 1 */
            issue(b + GS_DEPTH - 1, cn);   /* into step b - 1's buffer */
            columns(b + GS_DEPTH, cn);
            if (tid == 0) { /* in order, four values per shared-memory load */
                const uint32_t n = min(GS_STEP, je - (jb + b * GS_STEP));
                const float *sv = s_val[b % GS_DEPTH];
                uint32_t k = 0;
                for (; k + 4 <= n; k += 4) {
                    const float4 q = *(const float4 *)(sv + k);
                    sum += q.x;
                    sum += q.y;
                    sum += q.z;
                    sum += q.w;
                }
                for (; k < n; ++k) sum += sv[k];
            }
        }
        cp_async_wait<0>(); /* no copy in flight when the block leaves */
        if (tid == 0) gs_apply<EDGE, TRACK>(v, sum, outdeg, pr_new, val, delta, reset, damping);
        return;
    }
    if (blockIdx.x < nb + nwb) { /* warp class */
        const uint32_t i = wb + (blockIdx.x - nb) * 8 + warp;
        if (i >= bb) return;
        const uint32_t v = order[i];
        const uint32_t jb = rowptr[v], je = rowptr[v + 1];
        float sum = 0.0f;
        float x = jb + lane < je ? gs_in_value(__ldg(col + jb + lane), v, pr_old, pr_new) : 0.0f;
        for (uint32_t j0 = jb; j0 < je; j0 += 32) {
            const uint32_t nj = j0 + 32 + lane;
            const float y = nj < je ? gs_in_value(__ldg(col + nj), v, pr_old, pr_new) : 0.0f;
            const uint32_t n = min(32u, je - j0);
            for (uint32_t k = 0; k < n; ++k) {
                const float z = __shfl_sync(0xFFFFFFFFu, x, (int)k);
                sum += z; /* every lane keeps the same running sum, in order */
            }
            x = y;
        }
        if (lane == 0) gs_apply<EDGE, TRACK>(v, sum, outdeg, pr_new, val, delta, reset, damping);
        return;
    }
    /* thread class */
    const uint32_t nth = (gridDim.x - nb - nwb) * blockDim.x;
    for (uint32_t i = tb + (blockIdx.x - nb - nwb) * blockDim.x + tid; i < wb; i += nth) {
        const uint32_t v = order[i];
        const uint32_t jb = rowptr[v], je = rowptr[v + 1];
        float sum = 0.0f;
        for (uint32_t j0 = jb; j0 < je; j0 += 8) {
            float x[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = j0 + k < je ? gs_in_value(__ldg(col + j0 + k), v, pr_old, pr_new) : 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (j0 + k < je) sum += x[k];
        }
        gs_apply<EDGE, TRACK>(v, sum, outdeg, pr_new, val, delta, reset, damping);
    }
}

/* The sweep's sums of delta[] and |val[]|: each block adds a fixed slice in
 * FP64, the last block to finish adds the block sums in block order, logs
 * delta_log[k] = sum delta and res_log[k] = sum delta / sum |val| for the k-th
 * sweep (k = *slot, then advanced) and raises *done when the residual is <= tol. */
constexpr int DSUM_BLOCKS = 256;
__global__ void __launch_bounds__(256) k_gs_delta_sum(const float *__restrict__ delta, const float *__restrict__ val,
                                                      uint32_t nv, double2 *part, uint32_t *ticket, uint32_t *slot,
                                                      int *done, double tol, double *delta_log, double *res_log) {
    if (*(volatile const int *)done) return;
    __shared__ double2 s[8];
    __shared__ int s_last;
    const uint32_t per = (nv + gridDim.x - 1) / gridDim.x;
    const uint32_t b0 = blockIdx.x * per, b1 = min(nv, b0 + per);
    double x = 0.0, y = 0.0;
    for (uint32_t v = b0 + threadIdx.x; v < b1; v += blockDim.x) {
        x += (double)delta[v];
        y += fabs((double)val[v]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        y += __shfl_down_sync(0xFFFFFFFFu, y, o);
    }
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = make_double2(x, y);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < 8; ++w) {
            t.x += s[w].x;
            t.y += s[w].y;
        }
        part[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    double dx = 0.0, ny = 0.0;
    for (uint32_t b = 0; b < gridDim.x; ++b) {
        const double2 p = __ldcg(part + b);
        dx += p.x;
        ny += p.y;
    }
    const uint32_t k = *slot;
    const double res = ny > 0.0 ? dx / ny : 0.0;
    delta_log[k] = dx;
    res_log[k] = res;
    *slot = k + 1;
    if (tol > 0.0 && res <= tol) *done = 1;
    *ticket = 0u;
}

/* the vertex values before the first sweep, for the progress log: the edge-value
 * program's 0.15 (pagerank.cpp:84), the in-memory program's pr * outc = 1 (or
 * 0.15 without out-edges, pagerank.cpp:137-139) */
__global__ void k_gs_val_init(uint32_t nv, const uint32_t *__restrict__ outdeg, float reset, int edge, float *val) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        val[v] = (edge || outdeg[v] == 0) ? reset : 1.0f;
}

/* pagerank.cpp:140-143: the stored value is pr * outc on the last iteration */
__global__ void k_gs_final(uint32_t nv, const uint32_t *__restrict__ outdeg, const float *__restrict__ pr, float *out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t oc = outdeg[v];
        out[v] = oc > 0 ? __fmul_rn(pr[v], (float)oc) : pr[v];
    }
}

inline unsigned vgrid(uint32_t n) {
    uint64_t b = ((uint64_t)n + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * 16;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

/* Level schedule of the id-ordered dependency DAG: order[] (vertices by
 * (level, class, id)) and off[GS_CLASSES * l + c] = first index of class c of
 * level l, nlev levels. */
struct GsPlan {
    uint32_t nlev = 0;
    dbuf<uint32_t> order;
    std::vector<uint32_t> off;
};

void free_gs_plan(GsPlan *p) { delete p; }

static int build_gs_plan(gcg_graph *g, GsPlan &pl) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    tbuf<uint32_t> level, pending, pos, total;
    GCG_TRY(level.alloc(nv, s));
    GCG_TRY(pending.alloc(nv, s));
    GCG_TRY(pos.alloc(nv, s));
    GCG_TRY(total.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(level.get(), 0, (size_t)nv * 4, s));
    k_gs_pending<<<vgrid(nv), 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), nv, pending.get());
    GCG_TRY(scan_u32(pending.get(), pos.get(), nv, total.get(), s));
    uint32_t nfwd = 0;
    GCG_CUDA(cudaMemcpyAsync(&nfwd, total.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    uint32_t maxl = 0;
    if (nfwd) {
        /* the forward (u < v) edges grouped by source */
        tbuf<uint64_t> keys, tmp;
        tbuf<uint32_t> fwd_off, fwd_dst, front, cnt;
        GCG_TRY(keys.alloc(nfwd, s));
        GCG_TRY(tmp.alloc(nfwd, s));
        GCG_TRY(fwd_off.alloc((size_t)nv + 1, s));
        GCG_TRY(fwd_dst.alloc(nfwd, s));
        GCG_TRY(front.alloc((size_t)2 * nv, s));
        k_gs_fwd_keys<<<vgrid(nv), 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), nv, pending.get(), pos.get(),
                                                g->vbits, keys.get());
        uint64_t *sorted = nullptr;
        GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nfwd, (int)g->vbits, (int)(2 * g->vbits), &sorted, s));
        k_gs_fwd_off<<<vgrid(nfwd), 256, 0, s>>>(sorted, nfwd, g->vbits, nv, fwd_off.get(), fwd_dst.get());
        /* rounds, queued in batches of 64 (empty rounds return at once); the host
         * checks the last frontier count of each batch. A vertex joins a frontier
         * once, so at most nv rounds. */
        const uint32_t CAP = nv + 2;
        GCG_TRY(cnt.alloc(CAP, s));
        GCG_CUDA(cudaMemsetAsync(cnt.get(), 0, (size_t)CAP * 4, s));
        k_gs_roots<<<vgrid(nv), 256, 0, s>>>(pending.get(), nv, front.get(), cnt.get());
        GCG_LAUNCH_CHECK();
        uint32_t r = 0;
        for (;;) {
            const uint32_t nb = std::min<uint32_t>(64, CAP - 2 - r);
            for (uint32_t k = 0; k < nb; ++k, ++r) {
                uint32_t *cur = front.get() + (size_t)(r & 1) * nv, *nxt = front.get() + (size_t)((r + 1) & 1) * nv;
                k_gs_round<<<vgrid(nv), 256, 0, s>>>(r, fwd_off.get(), fwd_dst.get(), pending.get(), level.get(), cur,
                                                     nxt, cnt.get());
            }
            GCG_LAUNCH_CHECK();
            uint32_t last = 0;
            GCG_CUDA(cudaMemcpyAsync(&last, cnt.get() + r, 4, cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            if (last == 0 || r + 2 >= CAP) break;
        }
        /* the deepest non-empty round */
        std::vector<uint32_t> hc(r + 1);
        GCG_CUDA(cudaMemcpyAsync(hc.data(), cnt.get(), (size_t)(r + 1) * 4, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        uint64_t placed = 0;
        for (uint32_t k = 0; k <= r; ++k) {
            placed += hc[k];
            if (hc[k]) maxl = k;
        }
        if (placed != nv) return fail(GCG_ERR_CUDA, "level schedule: a vertex was not reached");
    }
    pl.nlev = maxl + 1;
    uint32_t lbits = 1;
    while (lbits < 32 && (1ull << lbits) <= maxl) ++lbits;
    if (g->vbits + 2 + lbits > 64) return fail(GCG_ERR_UNSUPPORTED, "level schedule: too many levels");
    tbuf<uint64_t> keys, tmp;
    GCG_TRY(keys.alloc(nv, s));
    GCG_TRY(tmp.alloc(nv, s));
    k_level_keys<<<vgrid(nv), 256, 0, s>>>(level.get(), g->in_rowptr.get(), nv, g->vbits, keys.get());
    uint64_t *sorted = nullptr;
    GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nv, (int)g->vbits, (int)(g->vbits + 2 + lbits), &sorted, s));
    const size_t nseg = (size_t)GS_CLASSES * pl.nlev;
    tbuf<uint32_t> doff;
    GCG_TRY(doff.alloc(nseg + 1, s));
    GCG_TRY(pl.order.alloc(nv));
    k_level_bounds<<<vgrid(nv), 256, 0, s>>>(sorted, nv, g->vbits, (uint32_t)nseg, doff.get(), pl.order.get());
    GCG_LAUNCH_CHECK();
    pl.off.resize(nseg + 1);
    GCG_CUDA(cudaMemcpyAsync(pl.off.data(), doff.get(), (nseg + 1) * 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    return GCG_OK;
}

/* GCG_PR_GS_EXACT (in-memory program) and GCG_PR_GS_EDGE (edge-value program).
 * With tol > 0, residuals or delta_log (always for GS_EDGE) every sweep also
 * tracks the vertices' pageranks: delta_log gets sum |pagerank - previous| and
 * residuals that sum over sum |pagerank| (the Jacobi residual's definition); the
 * run stops after the first sweep whose residual is <= tol. */
int pagerank_gs_exact(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    const bool edge = p->mode == GCG_PR_GS_EDGE;
    const bool track = edge || p->tol > 0.0 || p->residuals || p->delta_log;
    if (!g->gsplan) { /* built once per graph, dropped when its edges change */
        GsPlan *np = new GsPlan();
        const int st = build_gs_plan(g, *np);
        if (st != GCG_OK) {
            delete np;
            return st;
        }
        g->gsplan = np;
    }
    const GsPlan &pl = *g->gsplan;
    const int nsw = p->max_sweeps;
    tbuf<float> pr, val, delta;
    tbuf<double> logs; /* delta_log[nsw], res_log[nsw] */
    tbuf<double2> part;
    tbuf<uint32_t> ctl; /* ticket, slot, done */
    GCG_TRY(pr.alloc((size_t)2 * nv, s));
    GCG_TRY(ctl.alloc(4, s));
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 4 * sizeof(uint32_t), s));
    int *done = (int *)(ctl.get() + 2);
    float *pr_old = pr.get(), *pr_new = pr.get() + nv;
    const float reset = (float)p->teleport;
    if (track) {
        GCG_TRY(val.alloc(nv, s));
        GCG_TRY(delta.alloc(nv, s));
        GCG_TRY(logs.alloc(2 * (size_t)std::max(1, nsw), s));
        GCG_TRY(part.alloc(DSUM_BLOCKS, s));
        k_gs_val_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), reset, edge ? 1 : 0, val.get());
    }
    if (edge) k_gs_edge_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), pr_old);
    else k_gs_init<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), reset, pr_old);
    GCG_LAUNCH_CHECK();

    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    /* one sweep = all levels in order, then pr_old <- pr_new; captured once */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap;
    GCG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    GCG_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    for (uint32_t l = 0; l < pl.nlev; ++l) {
        const uint32_t *o = pl.off.data() + (size_t)GS_CLASSES * l;
        const uint32_t tb = o[0], wb = o[1], bb = o[2], be = o[3];
        if (tb == be) continue;
        /* blocks: one per block-class vertex, one per 8 warp-class vertices, then
         * the thread-class vertices (grid-strided) */
        const uint64_t nthr = wb - tb;
        const unsigned gr = (unsigned)((be - bb) + (bb - wb + 7) / 8 + (nthr ? vgrid((uint32_t)nthr) : 0));
        const uint32_t *rp = g->in_rowptr.get(), *cl = g->in_col.get(), *od = g->outdeg.get();
        if (edge)
            k_gs_level<true, true><<<gr, 256, 0, cap>>>(pl.order.get(), tb, wb, bb, be, rp, cl, od, pr_old, pr_new,
                                                        val.get(), delta.get(), done, p->teleport, p->damping);
        else if (track)
            k_gs_level<false, true><<<gr, 256, 0, cap>>>(pl.order.get(), tb, wb, bb, be, rp, cl, od, pr_old, pr_new,
                                                         val.get(), delta.get(), done, p->teleport, p->damping);
        else
            k_gs_level<false, false><<<gr, 256, 0, cap>>>(pl.order.get(), tb, wb, bb, be, rp, cl, od, pr_old, pr_new,
                                                          nullptr, nullptr, done, p->teleport, p->damping);
    }
    if (track)
        k_gs_delta_sum<<<DSUM_BLOCKS, 256, 0, cap>>>(delta.get(), val.get(), nv, part.get(), ctl.get(), ctl.get() + 1,
                                                     done, p->tol, logs.get(), logs.get() + std::max(1, nsw));
    cudaMemcpyAsync(pr_old, pr_new, (size_t)nv * 4, cudaMemcpyDeviceToDevice, cap);
    cudaError_t ce = cudaStreamEndCapture(cap, &graph);
    if (ce != cudaSuccess) {
        cudaStreamDestroy(cap);
        return fail(GCG_ERR_CUDA, std::string("sweep capture: ") + cudaGetErrorString(ce));
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaStreamDestroy(cap);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(GCG_ERR_CUDA, std::string("sweep graph instantiate: ") + cudaGetErrorString(ce));
    }
    /* sweeps are queued in chunks of 8; with a tolerance the host checks the
     * sweep count after each chunk (sweeps queued past convergence return at once) */
    uint32_t h_ctl[4] = {0, 0, 0, 0};
    GCG_CUDA(cudaEventRecord(ev0, s));
    for (int sw = 0; sw < nsw;) {
        const int n = std::min(8, nsw - sw);
        for (int k = 0; k < n; ++k) GCG_CUDA(cudaGraphLaunch(exec, s));
        sw += n;
        if (p->tol > 0.0 && sw < nsw) {
            GCG_CUDA(cudaMemcpyAsync(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            if (h_ctl[2]) break;
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaMemcpyAsync(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
    if (!edge) {
        k_gs_final<<<vgrid(nv), 256, 0, s>>>(nv, g->outdeg.get(), pr_old, pr_new);
        GCG_LAUNCH_CHECK();
    }
    GCG_CUDA(cudaEventSynchronize(ev1));
    GCG_CUDA(cudaStreamSynchronize(s));
    const int sweeps = track ? (int)h_ctl[1] : nsw;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    double last_res = 0.0;
    if (track && sweeps > 0)
        GCG_CUDA(cudaMemcpy(&last_res, logs.get() + std::max(1, nsw) + sweeps - 1, sizeof(double),
                            cudaMemcpyDeviceToHost));
    if (out_rank) GCG_TRY(copy_out(out_rank, edge ? val.get() : pr_new, (size_t)nv * 4, s));
    if (track && p->delta_log && sweeps > 0)
        GCG_TRY(copy_out(p->delta_log, logs.get(), (size_t)sweeps * sizeof(double), s));
    if (track && p->residuals && sweeps > 0)
        GCG_TRY(copy_out(p->residuals, logs.get() + std::max(1, nsw), (size_t)sweeps * sizeof(double), s));
    if (p->work_log && sweeps > 0) { /* every vertex updated per sweep; its in-edges (+ out-edges with edge values) */
        std::vector<uint64_t> wl(2 * (size_t)sweeps);
        for (int i = 0; i < sweeps; ++i) {
            wl[2 * i] = (uint64_t)nv * (uint64_t)(i + 1);
            wl[2 * i + 1] = (edge ? 2 : 1) * g->ne * (uint64_t)(i + 1);
        }
        GCG_TRY(copy_out(p->work_log, wl.data(), wl.size() * sizeof(uint64_t), s));
    }
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = (int)h_ctl[2];
        stats->residual = last_res;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = ms;
        stats->timed_sweeps = sweeps;
        stats->kernel_launches = 1 + (track ? 1 : 0) + (edge ? 0 : 1) + ((int)pl.nlev + (track ? 1 : 0)) * sweeps;
        stats->levels = (int)pl.nlev;
    }
    return GCG_OK;
}

}  // namespace gcg
