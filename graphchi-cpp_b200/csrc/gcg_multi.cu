/*
 * Many independent graphs, one persistent launch.
 *
 * The engine's addition for batches of uneven graphs (no reference counterpart:
 * the reference runs one graph per engine). gcg_batch_create concatenates the
 * graphs' in-CSRs into one block-diagonal union (vertex and edge offsets; each
 * graph is one interval) and builds the PageRank chunk plan on it, so the
 * out-degree relabelling and the shared-memory hub cache serve all graphs.
 *
 * gcg_batch_pagerank runs every sweep of every graph inside ONE cooperative
 * persistent kernel (one 1024-thread CTA per SM). Per sweep, four phases split by
 * a grid barrier:
 *   A  edges: warps stride over the 256-edge chunks of the still-active graphs
 *      (their concatenated chunk ranges; equal-sized chunks need no queue) and run
 *      the same pipelined gather / warp reduction as the single-graph kernel;
 *   B  rows crossing chunks: partials added in chunk order;
 *   C  vertices: CTAs pull 4096-row tiles (4 rows per thread) of the active graphs from a device work
 *      queue (atomic counter), apply, and write one FP64 residual partial per tile
 *      (fixed slot);
 *   D  one warp per graph adds its tile partials in a fixed order; a graph whose
 *      residual is <= tol (or that reached max_sweeps) leaves the queues.
 * The kernel ends when no graph is active. A whole solve (state init, initial
 * vector, the persistent kernel, rank assembly) is captured once into a CUDA
 * graph per parameter set and replayed; gcg_batch_autotune picks the hub-cache
 * size and the edge phase's work distribution by timing the candidates. Each graph's ranks are formed with the
 * same sums in the same order as its single-graph solve (only the FP64 residual
 * is reduced in a different order). Contributions change between
 * sweeps inside the kernel, so they are read with L2-coherent loads, never the
 * non-coherent path.
 *
 * Every grid-barrier wait is bounded: after the spin limit the kernel raises an
 * error flag and returns, and the host reports GCG_ERR_TIMEOUT.
 */
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"
#include "gcg_pr_device.cuh"

namespace gcg {
namespace {

constexpr uint32_t VROWS = 4;                 /* rows per thread in a vertex tile */
constexpr uint32_t VT = EDGE_THREADS * VROWS; /* rows per vertex tile */
constexpr uint32_t NG_MAX = 1024;     /* graphs per batch */
static_assert(NG_MAX <= EDGE_THREADS, "active_prefix gives each graph one thread of the CTA");

/* per-graph ranges in the union */
struct GRange {
    uint32_t cs, ce;      /* chunks [cs, ce) holding the graph's edges */
    uint32_t ss, se;      /* split-row list entries */
    uint32_t ns, ne;      /* rows with in-edges (nz index range) */
    uint32_t zs, ze;      /* rows without in-edges (zero index range) */
    uint32_t it_nz, it_z; /* first tile slot of its nz tiles / zero tiles */
    uint32_t gend;        /* end of the graph's edges in the union (its chunks stop there) */
    uint32_t pad1;
};

struct MultiArgs {
    SweepArgs a;            /* union graph arguments (buffers set per sweep inside) */
    float *c[2];
    float *rnz[2];
    const GRange *gr;
    uint32_t ng, max_sweeps;
    double2 *tile_part;     /* per tile slot */
    const double *norm_const; /* per graph */
    int *active;            /* per graph */
    int *gsweeps;           /* per graph: sweeps run */
    double *gres;           /* per graph: last residual */
    uint32_t *qctr;         /* [2 parities][2 queues] */
    uint32_t *bar;          /* [0] arrivals, [1] generation */
    int *err;
    long long spin_limit;
    uint32_t extra_arrivals; /* test hook: the barrier waits for this many more CTAs */
    uint32_t grab;           /* edge phase without per-graph hubs: 0 = warps stride over the chunks;
                                g > 0 = warps take runs of g chunks from a device work queue */
    const uint32_t *voff;    /* per-graph hubs: first union vertex of each graph (ng + 1
                                entries), NULL = one hub over the union's hottest sources */
    const uint32_t *long_g;  /* graph of each long split row (a.long_split order) */
    uint32_t nlong;
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/* Grid barrier with a bounded wait; returns false (all CTAs) once any CTA timed out. */
__device__ bool grid_sync(const MultiArgs &m, uint32_t &gen) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t target = gen + 1;
        const uint32_t expect = gridDim.x + m.extra_arrivals;
        if (atomicAdd(m.bar, 1u) == expect - 1) {
            atomicExch(m.bar, 0u);
            __threadfence();
            atomicExch(m.bar + 1, target);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(m.bar + 1) < target) {
                if (*(volatile int *)m.err || ++spins > m.spin_limit) {
                    atomicExch(m.err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        gen = target;
        __threadfence();
        s_ok = *(volatile int *)m.err == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

/* smallest range of chunks a CTA takes at a time in the edge phase with
 * per-graph hubs (two per warp of the CTA) */
constexpr uint32_t GRAB_MIN = 64;

/* Exclusive prefix over the active graphs of a per-graph count (which: 0 edge
 * chunks, 1 split rows, 2 vertex tiles), in shared memory: thread g of the CTA
 * reads graph g's flag and range (ng <= the block size), a block-wide scan adds
 * them up. *nactive receives the number of active graphs. Every CTA computes
 * the same prefix: the flags change only between grid barriers. */
__device__ uint32_t active_prefix(const MultiArgs &m, int which, uint32_t *s_pref, int const_pass,
                                  uint32_t *nactive = nullptr, uint32_t *s_cs = nullptr) {
    __shared__ uint32_t s_wsum[EDGE_THREADS / 32];
    const uint32_t g = threadIdx.x, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t cnt = 0;
    int act = 0;
    if (s_cs && g < m.ng) { /* chunk range of every graph, for the edge phase: [s_cs[g], s_cs[g + 1]) */
        const GRange r = m.gr[g];
        s_cs[g] = r.cs;
        if (g + 1 == m.ng) s_cs[m.ng] = r.ce;
    }
    if (g < m.ng && *(volatile const int *)(m.active + g)) {
        act = 1;
        const GRange r = m.gr[g];
        cnt = which == 0 ? r.ce - r.cs
            : which == 1 ? r.se - r.ss
                         : (r.ne - r.ns + VT - 1) / VT + (const_pass ? (r.ze - r.zs + VT - 1) / VT : 0u);
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= (uint32_t)d) incl += y;
    }
    if (lane == 31) s_wsum[warp] = incl;
    const int na = __syncthreads_count(act);
    if (warp == 0) {
        const uint32_t w = lane < blockDim.x / 32 ? s_wsum[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, d);
            if (lane >= (uint32_t)d) wi += y;
        }
        if (lane < blockDim.x / 32) s_wsum[lane] = wi - w; /* exclusive warp offsets */
    }
    __syncthreads();
    const uint32_t excl = incl - cnt + s_wsum[warp];
    if (g < m.ng) s_pref[g] = excl;
    if (g + 1 == m.ng) s_pref[m.ng] = excl + cnt;
    __syncthreads();
    if (nactive) *nactive = (uint32_t)na;
    return s_pref[m.ng];
}

/* the active graph whose range holds position x of the concatenation */
__device__ __forceinline__ uint32_t find_graph(const uint32_t *s_pref, uint32_t ng, uint32_t x) {
    uint32_t lo = 0, hi = ng; /* largest g with s_pref[g] <= x: its range is non-empty */
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_pref[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

/* PG: per-graph hubs (m.voff set), else one hub over the union's hottest sources */
template <bool PG>
__global__ void __launch_bounds__(EDGE_THREADS, 1) k_multi_pagerank(MultiArgs m) {
    extern __shared__ float s_hub[];
    __shared__ uint32_t s_pref[NG_MAX + 1];
    __shared__ uint32_t s_cs[NG_MAX + 1];
    __shared__ uint32_t s_item, s_grab;
    __shared__ double2 s_red[EDGE_THREADS / 32];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint64_t pol_stream = policy_evict_first(), pol_keep = policy_evict_last();
    uint32_t gen = 0;
    SweepArgs a = m.a;

    for (uint32_t sweep = 0; sweep < m.max_sweeps; ++sweep) {
        a.c_old = m.c[sweep & 1];
        a.c_new = m.c[(sweep + 1) & 1];
        a.r_nz_old = m.rnz[sweep & 1];
        a.r_nz_new = m.rnz[(sweep + 1) & 1];
        const int const_pass = sweep < 2;
        uint32_t *qC = m.qctr + 2 * (sweep & 1) + 1;

        /* ---- A: edge chunks of the active graphs, grid-strided over their
         *         concatenation (chunks are equal-sized), loads one chunk ahead ---- */
        uint32_t nact = 0;
        const uint32_t totA = active_prefix(m, 0, s_pref, const_pass, &nact, s_cs);
        if (nact == 0) break; /* every graph has stopped: the same answer in every CTA */
        if (PG) {
            /* Per-graph hubs: every graph's sources are relabelled by out-degree
             * within its own id range, so a graph's hottest sources are the first
             * ids of its range. CTAs take ranges of the active graphs' chunks (in
             * graph order) from a device cursor, guided: a grab is 1/(2 x CTAs) of
             * what is left, at least GRAB_MIN chunks, so early grabs are large and
             * the last ones small. For each graph a range touches, the CTA loads
             * that graph's hub into shared memory (unless it holds it already) and
             * its warps stride over the graph's chunks, one chunk loaded ahead. */
            uint32_t *cursor = m.qctr + 2 * (sweep & 1);
            uint32_t cur = 0xFFFFFFFFu, hb = 0, hn = 0;
            for (;;) {
                if (threadIdx.x == 0) {
                    const uint32_t seen = *(volatile uint32_t *)cursor;
                    const uint32_t left = seen < totA ? totA - seen : 0u;
                    const uint32_t want = max(GRAB_MIN, left / (2u * gridDim.x));
                    s_item = atomicAdd(cursor, want);
                    s_grab = want;
                }
                __syncthreads(); /* also: every warp is done with the previous range */
                const uint32_t lo = s_item, hi = min(totA, lo + s_grab);
                __syncthreads();
                if (lo >= totA) break;
                for (uint32_t x = lo; x < hi;) {
                    const uint32_t g = find_graph(s_pref, m.ng, x);
                    const uint32_t send = min(hi, s_pref[g + 1]);
                    if (g != cur) {
                        if (x != lo) __syncthreads(); /* the previous graph's gathers are done */
                        const uint32_t v0 = m.voff[g], v1 = m.voff[g + 1];
                        hb = v0 & ~3u;                      /* 16-byte aligned start */
                        hn = min(a.hub + (v0 - hb), v1 - hb); /* entries [hb, hb + hn) */
                        const float4 *src4 = (const float4 *)(a.c_old + hb);
                        float4 *dst4 = (float4 *)s_hub;
                        const uint32_t n4 = hn >> 2;
                        for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) dst4[i] = __ldcg(src4 + i);
                        for (uint32_t i = (n4 << 2) + threadIdx.x; i < hn; i += blockDim.x)
                            s_hub[i] = __ldcg(a.c_old + hb + i);
                        __syncthreads();
                        cur = g;
                    }
                    const uint32_t cs0 = s_cs[g] - s_pref[g]; /* chunk = cs0 + position */
                    uint32_t col[EPL], flags = 0, nvalid = 0, base = 0;
                    uint32_t pos = x + warp;
                    if (pos < send) load_chunk(a, cs0 + pos, lane, pol_stream, col, flags, nvalid, base, a.ne);
                    while (pos < send) {
                        float val[EPL];
#pragma unroll
                        for (int j = 0; j < EPL; ++j) {
                            const uint32_t d = col[j] - hb;
                            float v = 0.0f;
                            if ((uint32_t)j < nvalid)
                                v = d < hn ? s_hub[d] : ld_cg_keep_f32(a.c_old + col[j], pol_keep);
                            val[j] = v;
                        }
                        const uint32_t cch = cs0 + pos, cf = flags, cn = nvalid, cb = base;
                        pos += EDGE_THREADS / 32;
                        if (pos < send) load_chunk(a, cs0 + pos, lane, pol_stream, col, flags, nvalid, base, a.ne);
                        reduce_chunk(a, cch, lane, val, cf, cn, cb, a.ne);
                    }
                    x = send;
                }
            }
        } else {
            /* one hub over the union's hottest sources */
            load_hub(a, s_hub);
            __syncthreads();
            /* runs of chunks: [item, item_end) is this warp's current run; the
             * next chunk is loaded while the current one is gathered */
            const uint32_t run = m.grab ? m.grab : 1u;
            uint32_t item, item_end;
            auto next_run = [&](uint32_t &it, uint32_t &end) {
                if (m.grab) {
                    uint32_t x = 0;
                    if (lane == 0) x = atomicAdd(m.qctr + 2 * (sweep & 1), run);
                    it = __shfl_sync(FULL, x, 0);
                } else {
                    it = (it == 0xFFFFFFFFu) ? gwarp : it + nwarps - 1u; /* it was incremented past its run of 1 */
                }
                end = it < totA ? (totA - it < run ? totA : it + run) : it;
            };
            item = 0xFFFFFFFFu;
            next_run(item, item_end);
            /* A graph's last chunk may end in filler edges: they form the row of
             * the graph's padding vertex (its own head, never read), so chunks
             * are reduced up to the union's end like the single-graph kernel's */
            uint32_t col[EPL], flags = 0, nvalid = 0, base = 0, ch = 0;
            auto load_item = [&](uint32_t it) {
                const uint32_t g = find_graph(s_pref, m.ng, it);
                ch = s_cs[g] + (it - s_pref[g]);
                load_chunk(a, ch, lane, pol_stream, col, flags, nvalid, base, a.ne);
            };
            if (item < item_end) load_item(item);
            while (item < item_end) {
                float val[EPL];
                gather_chunk<true>(a, col, nvalid, s_hub, pol_keep, val);
                const uint32_t cch = ch, cf = flags, cn = nvalid, cb = base;
                ++item;
                if (item >= item_end) next_run(item, item_end);
                if (item < item_end) load_item(item);
                reduce_chunk(a, cch, lane, val, cf, cn, cb, a.ne);
            }
        }
        if (!grid_sync(m, gen)) return;

        /* ---- B: rows crossing chunk boundaries, summed exactly as the
         *         single-graph fix-up does (k_pr_fix): long rows one per warp over
         *         the grid in the fixed group order of long_row_sum_warp (rows
         *         in relabelled order put a graph's long rows next to each other),
         *         short rows by one lane in chunk order ---- */
        for (uint32_t k = gwarp; k < m.nlong; k += nwarps) {
            const uint32_t g = m.long_g[k];
            if (g >= m.ng || !*(volatile const int *)(m.active + g)) continue;
            const uint4 sp = a.split[a.long_split[k]];
            const float s = long_row_sum_warp<true>(a.head_part, sp.y, sp.z, lane);
            if (lane == 0) a.nzsum[sp.x] = __ldcg(a.tail_part + sp.y) + s;
        }
        const uint32_t totB = active_prefix(m, 1, s_pref, const_pass);
        for (uint32_t wb = gwarp * 32u; wb < totB; wb += nwarps * 32u) {
            const uint32_t x = wb + lane;
            uint4 sp = make_uint4(0, 0, 0, 0);
            const bool valid = x < totB;
            if (valid) {
                const uint32_t g = find_graph(s_pref, m.ng, x);
                sp = a.split[m.gr[g].ss + (x - s_pref[g])];
            }
            if (valid && (sp.z - sp.y) <= LONG_SPAN) {
                float s = __ldcg(a.tail_part + sp.y);
                for (uint32_t c = sp.y + 1; c <= sp.z; ++c) s += __ldcg(a.head_part + c);
                a.nzsum[sp.x] = s;
            }
        }
        if (!grid_sync(m, gen)) return;

        /* ---- C: vertex tiles of the active graphs (work queue), one residual
         *         partial per tile ---- */
        const uint32_t totC = active_prefix(m, 2, s_pref, const_pass);
        for (;;) {
            if (threadIdx.x == 0) s_item = atomicAdd(qC, 1u);
            __syncthreads();
            const uint32_t item = s_item;
            __syncthreads();
            if (item >= totC) break;
            const uint32_t g = find_graph(s_pref, m.ng, item);
            const GRange r = m.gr[g];
            const uint32_t t = item - s_pref[g];
            const uint32_t ntn = (r.ne - r.ns + VT - 1) / VT;
            double d = 0.0, n = 0.0;
            uint32_t slot;
            if (t < ntn) {
                slot = r.it_nz + t;
                /* VROWS rows per thread (coalesced per row step), all loads first */
                const uint32_t i0 = r.ns + t * VT + threadIdx.x;
                float sum[VROWS], ro[VROWS];
                uint32_t od[VROWS], cid[VROWS];
#pragma unroll
                for (uint32_t u = 0; u < VROWS; ++u) {
                    const uint32_t i = i0 + u * EDGE_THREADS;
                    if (i < r.ne) {
                        sum[u] = __ldcg(a.nzsum + i);
                        ro[u] = __ldcg(a.r_nz_old + i);
                        od[u] = a.od_nz[i];
                        cid[u] = a.nz_cidx[i];
                    }
                }
#pragma unroll
                for (uint32_t u = 0; u < VROWS; ++u) {
                    const uint32_t i = i0 + u * EDGE_THREADS;
                    if (i < r.ne) {
                        const float rn = pr_value(a, sum[u]);
                        a.r_nz_new[i] = rn;
                        a.c_new[cid[u]] = od[u] ? __fdiv_rn(rn, (float)od[u]) : 0.0f;
                        d += fabs((double)rn - (double)ro[u]);
                        n += fabs((double)rn);
                    }
                }
            } else {
                slot = r.it_z + (t - ntn);
                for (uint32_t u = 0; u < VROWS; ++u) {
                    const uint32_t i = r.zs + (t - ntn) * VT + u * EDGE_THREADS + threadIdx.x;
                    if (i < r.ze) {
                        const uint32_t v = a.zero_rows[i];
                        const float rn = pr_value(a, 0.0f);
                        const float ro = sweep == 0 ? __ldcg(a.r_init + v) : rn;
                        const uint32_t od = a.outdeg[v];
                        a.c_new[a.zero_cidx[i]] = od ? __fdiv_rn(rn, (float)od) : 0.0f;
                        d += fabs((double)rn - (double)ro);
                        n += fabs((double)rn);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                d += __shfl_down_sync(FULL, d, o);
                n += __shfl_down_sync(FULL, n, o);
            }
            if (lane == 0) s_red[warp] = make_double2(d, n);
            __syncthreads();
            if (threadIdx.x == 0) {
                double2 tot = make_double2(0.0, 0.0);
                for (uint32_t w = 0; w < EDGE_THREADS / 32; ++w) {
                    tot.x += s_red[w].x;
                    tot.y += s_red[w].y;
                }
                m.tile_part[slot] = tot;
            }
        }
        if (!grid_sync(m, gen)) return;

        /* ---- D: per-graph residual and stop ---- */
        for (uint32_t g = gwarp; g < m.ng; g += nwarps) {
            if (!*(volatile int *)(m.active + g)) continue;
            const GRange r = m.gr[g];
            const uint32_t nt = (r.ne - r.ns + VT - 1) / VT;
            const uint32_t nz = const_pass ? (r.ze - r.zs + VT - 1) / VT : 0u;
            double d = 0.0, n = 0.0;
            for (uint32_t t = lane; t < nt + nz; t += 32u) {
                const double2 p = __ldcg(m.tile_part + (t < nt ? r.it_nz + t : r.it_z + (t - nt)));
                d += p.x;
                n += p.y;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                d += __shfl_xor_sync(FULL, d, o);
                n += __shfl_xor_sync(FULL, n, o);
            }
            if (lane == 0) {
                if (!const_pass) n += m.norm_const[g];
                const double res = n > 0.0 ? d / n : 0.0;
                m.gres[g] = res;
                m.gsweeps[g] = (int)sweep + 1;
                if ((a.tol > 0.0 && res <= a.tol) || sweep + 1 >= m.max_sweeps) m.active[g] = 0;
            }
        }
        /* the queues of the next sweep's parity were last used a sweep ago */
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            m.qctr[2 * ((sweep + 1) & 1)] = 0u;
            m.qctr[2 * ((sweep + 1) & 1) + 1] = 0u;
        }
        if (!grid_sync(m, gen)) return;
    }
}

/* result assembly: ranks of every vertex of every graph, from the buffer of the
 * sweep count its graph stopped at */
__global__ void k_multi_scatter(const GRange *__restrict__ gr, uint32_t ng, const int *__restrict__ gsweeps,
                                const uint32_t *__restrict__ nz_rows, const uint32_t *__restrict__ zero_rows,
                                const float *__restrict__ rnz0, const float *__restrict__ rnz1, float t,
                                float *__restrict__ r) {
    for (uint32_t g = blockIdx.y; g < ng; g += gridDim.y) {
        const GRange x = gr[g];
        const int sw = gsweeps[g];
        if (sw == 0) continue; /* no sweep: the initial vector stays */
        const float *src = (sw & 1) ? rnz1 : rnz0;
        for (uint32_t i = x.ns + blockIdx.x * blockDim.x + threadIdx.x; i < x.ne; i += gridDim.x * blockDim.x)
            r[nz_rows[i]] = src[i];
        for (uint32_t i = x.zs + blockIdx.x * blockDim.x + threadIdx.x; i < x.ze; i += gridDim.x * blockDim.x)
            r[zero_rows[i]] = t;
    }
}

__global__ void k_concat(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col,
                         const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ outdeg, uint32_t nv,
                         uint64_t ne, uint32_t voff, uint32_t eoff, uint32_t *__restrict__ urowptr,
                         uint32_t *__restrict__ ucol, uint32_t *__restrict__ uindeg, uint32_t *__restrict__ uoutdeg) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v <= nv; v += nth) {
        urowptr[voff + v] = rowptr[v] + eoff;
        if (v < nv) {
            uindeg[voff + v] = indeg[v];
            uoutdeg[voff + v] = outdeg[v];
        }
    }
    for (uint64_t e = tid; e < ne; e += nth) ucol[eoff + e] = col[e] + voff;
}

/* the padding vertex after a graph: in-edges [pe0, pe1) from itself, no out-edges */
__global__ void k_pad(uint32_t pv, uint32_t pe0, uint32_t pe1, uint32_t *__restrict__ urowptr, uint32_t *__restrict__ ucol,
                      uint32_t *__restrict__ uindeg, uint32_t *__restrict__ uoutdeg) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (tid == 0) {
        urowptr[pv] = pe0;
        urowptr[pv + 1] = pe1;
        uindeg[pv] = pe1 - pe0;
        uoutdeg[pv] = 0u;
    }
    for (uint32_t e = pe0 + tid; e < pe1; e += nth) ucol[e] = pv;
}

/* per-graph state at the start of a solve (on the device, so a whole solve can be
 * captured in a CUDA graph): all graphs active, counters clear, and the rank mass
 * of the vertices without in-edges (constant after the first sweep) */
__global__ void k_multi_init(const GRange *__restrict__ gr, uint32_t ng, double teleport,
                             double *__restrict__ norm_const, int *__restrict__ active, int *__restrict__ gsweeps,
                             double *__restrict__ gres, int *__restrict__ err, uint32_t *__restrict__ qctr,
                             uint32_t *__restrict__ bar) {
    const double t = fabs((double)(float)teleport);
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        norm_const[g] = (double)(gr[g].ze - gr[g].zs) * t;
        active[g] = 1;
        gsweeps[g] = 0;
        gres[g] = 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x < 4) qctr[threadIdx.x] = 0u;
    if (blockIdx.x == 0 && threadIdx.x < 2) bar[threadIdx.x] = 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0;
}

/* graph g's vertices keep their order at union offset voff[g]; map both ways */
__global__ void k_expand(const float *__restrict__ src, const uint32_t *__restrict__ roff, const uint32_t *__restrict__ voff,
                         uint32_t ng, float *__restrict__ dst, int to_union) {
    for (uint32_t g = blockIdx.y; g < ng; g += gridDim.y) {
        const uint32_t n = roff[g + 1] - roff[g];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            if (to_union) dst[voff[g] + i] = src[roff[g] + i];
            else dst[roff[g] + i] = src[voff[g] + i];
        }
    }
}

/* lower bound of each query id in a sorted id list */
__global__ void k_bounds(const uint32_t *__restrict__ ids, uint32_t n, const uint32_t *__restrict__ q, uint32_t nq,
                         uint32_t *__restrict__ out) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nq) return;
    const uint32_t x = q[g];
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ids[mid] < x) lo = mid + 1; else hi = mid;
    }
    out[g] = lo;
}

/* lower bound of each graph's first nz index in the split-row list */
__global__ void k_split_bounds(const uint4 *__restrict__ split, uint32_t n, const uint32_t *__restrict__ nzb, uint32_t nq,
                               uint32_t *__restrict__ out) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nq) return;
    const uint32_t x = nzb[g];
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (split[mid].x < x) lo = mid + 1; else hi = mid;
    }
    out[g] = lo;
}

}  // namespace
}  // namespace gcg

/* ---- host side ------------------------------------------------------------ */

struct gcg_batch {
    uint32_t ng = 0;
    gcg_graph *u = nullptr; /* the union graph (owned) */
    std::vector<uint32_t> voff, eoff;   /* union vertex / edge offset of each graph (edges 256-aligned) */
    std::vector<uint32_t> roff;         /* offset of each graph in the callers' arrays (no padding) */
    std::vector<gcg::GRange> gr_host;
    gcg::dbuf<uint32_t> d_roff, d_voff;
    gcg::dbuf<uint32_t> long_g; /* graph of each long split row of the union (or ng: none) */
    uint32_t ntiles = 0;
    gcg::dbuf<gcg::GRange> gr;
    /* workspace, allocated on the first solve */
    gcg::dbuf<float> c, rnz, r, nzsum, parts;
    gcg::dbuf<double2> tile_part;
    gcg::dbuf<double> norm_const, gres;
    gcg::dbuf<int> active, gsweeps, err;
    gcg::dbuf<uint32_t> qctr, bar;
    gcg::dbuf<float> rout; /* ranks in the callers' layout */
    /* launch configuration (gcg_batch_autotune): shared-memory hub entries
     * (UINT32_MAX = the plan's), edge-phase queue run length (0 = strided) */
    uint32_t tune_hub = 0xFFFFFFFFu, tune_grab = 0;
    /* the captured solve, replayed while the parameters stay the same */
    cudaGraphExec_t gexec = nullptr;
    bool graph_unsupported = false;
    double key_t = 0, key_d = 0, key_tol = 0;
    int key_ms = -1;
    float key_init = 0;
    uint32_t key_hub = 0, key_grab = 0;
    /* the batch's own stream (capturable), used until the caller sets one; it
     * waits for the legacy default stream at the start of every solve */
    cudaStream_t own = nullptr;
    ~gcg_batch() {
        if (gexec) cudaGraphExecDestroy(gexec);
        delete u;
        if (own) cudaStreamDestroy(own);
    }
};

namespace gcg {

static int batch_build(gcg_graph *const *graphs, uint32_t ng, uint32_t flags, gcg_batch *b) {
    b->ng = ng;
    b->voff.assign(ng + 1, 0);
    b->eoff.assign(ng + 1, 0);
    b->roff.assign(ng + 1, 0);
    std::vector<uint32_t> gend(ng);
    uint64_t V = 0, E = 0, R = 0;
    for (uint32_t g = 0; g < ng; ++g) {
        E = (E + CH - 1) / CH * CH; /* the graph starts on a chunk boundary */
        b->voff[g] = (uint32_t)V;
        b->eoff[g] = (uint32_t)E;
        b->roff[g] = (uint32_t)R;
        V += graphs[g]->nv + 1; /* + its padding vertex */
        R += graphs[g]->nv;
        E += graphs[g]->ne;
        gend[g] = (uint32_t)E;
        if (V > MAX_VERTICES || E + CH > MAX_EDGES)
            return fail(GCG_ERR_UNSUPPORTED, "gcg_batch_create: more than 2^32 - 2^26 vertices or edges in total");
    }
    const uint64_t Etot = (E + CH - 1) / CH * CH;
    b->voff[ng] = (uint32_t)V;
    b->eoff[ng] = (uint32_t)Etot;
    b->roff[ng] = (uint32_t)R;
    gcg_graph *u = new gcg_graph();
    b->u = u;
    u->nv = (uint32_t)V;
    u->ne = Etot;
    u->vbits = 1;
    while (u->vbits < 32 && (1ull << u->vbits) < V) ++u->vbits;
    if (u->in_rowptr.alloc((size_t)V + 1) || u->in_col.alloc(Etot) || u->indeg.alloc(V) || u->outdeg.alloc(V))
        return GCG_ERR_NOMEM;
    for (uint32_t g = 0; g < ng; ++g) {
        const gcg_graph *x = graphs[g];
        const uint64_t n = std::max<uint64_t>(x->nv + 1ull, x->ne);
        const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)num_sms() * 16));
        k_concat<<<blocks, 256>>>(x->in_rowptr.get(), x->in_col.get(), x->indeg.get(), x->outdeg.get(), x->nv, x->ne,
                                  b->voff[g], b->eoff[g], u->in_rowptr.get(), u->in_col.get(), u->indeg.get(),
                                  u->outdeg.get());
        /* padding vertex: the filler edges up to the next graph's chunk boundary */
        k_pad<<<8, 256>>>(b->voff[g] + x->nv, gend[g], b->eoff[g + 1], u->in_rowptr.get(), u->in_col.get(),
                          u->indeg.get(), u->outdeg.get());
    }
    GCG_LAUNCH_CHECK();
    /* each graph (with its padding vertex) is one interval of the union */
    u->nshards = ng;
    GCG_TRY(u->intervals_dev.alloc(ng));
    u->intervals_host = (uint32_t *)malloc((size_t)ng * 4);
    for (uint32_t g = 0; g < ng; ++g) u->intervals_host[g] = b->voff[g + 1] - 1;
    GCG_CUDA(cudaMemcpy(u->intervals_dev.get(), u->intervals_host, (size_t)ng * 4, cudaMemcpyHostToDevice));
    u->union_of_graphs = true;
    /* by default every graph keeps its id range: per-graph hubs */
    u->relabel_per_interval = (flags & GCG_BATCH_ONE_HUB) == 0;
    GCG_TRY(ensure_chunk_plan(u));
    const ChunkPlan &pl = *u->cplan;
    /* per-graph ranges (padding vertices excluded) by binary search on the device:
     * query 2g = first vertex of graph g, 2g+1 = its padding vertex. The plan's
     * rows are in relabelled order, which keeps every graph's id range and puts
     * the padding vertex (no out-edges, the range's largest id) last, so the
     * search runs on the relabelled ids (on the original ids for a union whose
     * rows kept the original order) */
    const uint32_t nq = 2 * ng;
    std::vector<uint32_t> q(nq);
    for (uint32_t g = 0; g < ng; ++g) {
        q[2 * g] = b->voff[g];
        q[2 * g + 1] = b->voff[g] + graphs[g]->nv;
    }
    dbuf<uint32_t> dq, nzb, zb, sb;
    GCG_TRY(dq.alloc(nq));
    GCG_TRY(nzb.alloc(nq));
    GCG_TRY(zb.alloc(nq));
    GCG_TRY(sb.alloc(nq));
    GCG_CUDA(cudaMemcpy(dq.get(), q.data(), nq * 4, cudaMemcpyHostToDevice));
    const unsigned gb = (nq + 255) / 256;
    k_bounds<<<gb, 256>>>(pl.rows_relabelled ? pl.nz_cidx.get() : pl.nz_rows.get(), pl.nnz, dq.get(), nq, nzb.get());
    k_bounds<<<gb, 256>>>(pl.rows_relabelled ? pl.zero_cidx.get() : pl.zero_rows.get(), pl.nzero, dq.get(), nq,
                          zb.get());
    k_split_bounds<<<gb, 256>>>(pl.split.get(), pl.nsplit, nzb.get(), nq, sb.get());
    GCG_LAUNCH_CHECK();
    std::vector<uint32_t> hn(nq), hz(nq), hs(nq);
    GCG_CUDA(cudaMemcpy(hn.data(), nzb.get(), nq * 4, cudaMemcpyDeviceToHost));
    GCG_CUDA(cudaMemcpy(hz.data(), zb.get(), nq * 4, cudaMemcpyDeviceToHost));
    GCG_CUDA(cudaMemcpy(hs.data(), sb.get(), nq * 4, cudaMemcpyDeviceToHost));
    b->gr_host.resize(ng);
    uint32_t tiles = 0;
    for (uint32_t g = 0; g < ng; ++g) {
        GRange &r = b->gr_host[g];
        r.cs = b->eoff[g] / CH;
        r.ce = (gend[g] + CH - 1) / CH;
        r.gend = gend[g];
        r.ns = hn[2 * g];
        r.ne = hn[2 * g + 1];
        r.zs = hz[2 * g];
        r.ze = hz[2 * g + 1];
        r.ss = hs[2 * g];
        r.se = hs[2 * g + 1];
        r.it_nz = tiles;
        tiles += (r.ne - r.ns + VT - 1) / VT;
        r.it_z = tiles;
        tiles += (r.ze - r.zs + VT - 1) / VT;
        r.pad1 = 0;
    }
    b->ntiles = tiles;
    /* the graph of each long split row (the padding rows never span that far) */
    {
        std::vector<uint32_t> ls(pl.nlong), lg(std::max<uint32_t>(pl.nlong, 1), ng);
        if (pl.nlong)
            GCG_CUDA(cudaMemcpy(ls.data(), pl.long_split.get(), (size_t)pl.nlong * 4, cudaMemcpyDeviceToHost));
        for (uint32_t k = 0; k < pl.nlong; ++k) {
            uint32_t lo = 0, hi = ng; /* last graph whose split range starts at or before ls[k] */
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (b->gr_host[mid].ss <= ls[k]) lo = mid; else hi = mid;
            }
            if (b->gr_host[lo].ss <= ls[k] && ls[k] < b->gr_host[lo].se) lg[k] = lo;
        }
        GCG_TRY(b->long_g.alloc(lg.size()));
        GCG_CUDA(cudaMemcpy(b->long_g.get(), lg.data(), lg.size() * 4, cudaMemcpyHostToDevice));
    }
    GCG_TRY(b->gr.alloc(ng));
    GCG_CUDA(cudaMemcpy(b->gr.get(), b->gr_host.data(), ng * sizeof(GRange), cudaMemcpyHostToDevice));
    GCG_TRY(b->d_roff.alloc(ng + 1));
    GCG_TRY(b->d_voff.alloc(ng + 1));
    GCG_CUDA(cudaMemcpy(b->d_roff.get(), b->roff.data(), (ng + 1) * 4, cudaMemcpyHostToDevice));
    GCG_CUDA(cudaMemcpy(b->d_voff.get(), b->voff.data(), (ng + 1) * 4, cudaMemcpyHostToDevice));
    return GCG_OK;
}

/* Enqueues one whole solve on the batch stream: per-graph state, initial vector,
 * the cooperative persistent kernel, the rank assembly and the map to the
 * callers' layout. Stream-ordered only (no host synchronisation), so it can be
 * captured into a CUDA graph. */
static int enqueue_solve(gcg_batch *b, MultiArgs &m, const gcg_pr_params *p, const float *init_dev, unsigned grid,
                         uint32_t hub_bytes) {
    gcg_graph *u = b->u;
    const ChunkPlan &pl = *u->cplan;
    const uint32_t ng = b->ng, nv = u->nv, nreal = b->roff[ng];
    cudaStream_t s = u->stream;
    k_multi_init<<<(ng + 255) / 256, 256, 0, s>>>(b->gr.get(), ng, p->teleport, b->norm_const.get(), b->active.get(),
                                                  b->gsweeps.get(), b->gres.get(), b->err.get(), b->qctr.get(),
                                                  b->bar.get());
    GCG_TRY(pr_init_state(u, p->init, init_dev, b->r.get(), b->c.get(), b->rnz.get()));
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(EDGE_THREADS);
    cfg.dynamicSmemBytes = hub_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t le = m.voff ? cudaLaunchKernelEx(&cfg, k_multi_pagerank<true>, m)
                            : cudaLaunchKernelEx(&cfg, k_multi_pagerank<false>, m);
    if (le != cudaSuccess)
        return fail(GCG_ERR_CUDA, std::string("gcg_batch_pagerank: cooperative launch: ") + cudaGetErrorString(le));
    dim3 sg((unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nv / ng + 255) / 256, 64)),
            std::min<uint32_t>(ng, 1024));
    k_multi_scatter<<<sg, 256, 0, s>>>(b->gr.get(), ng, b->gsweeps.get(), pl.nz_rows.get(), pl.zero_rows.get(),
                                       m.rnz[0], m.rnz[1], (float)p->teleport, b->r.get());
    const dim3 eg((unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nreal / ng + 255) / 256, 64)),
                  std::min<uint32_t>(ng, 1024));
    k_expand<<<eg, 256, 0, s>>>(b->r.get(), b->d_roff.get(), b->d_voff.get(), ng, b->rout.get(), 0);
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

static int batch_pagerank(gcg_batch *b, const gcg_pr_params *p, float *out, int32_t *sweeps, double *residuals,
                          gcg_pr_stats *stats, bool allow_graph = true) {
    gcg_graph *u = b->u;
    const ChunkPlan &pl = *u->cplan;
    const uint32_t nv = u->nv, ng = b->ng;
    cudaStream_t s = u->stream;
    if (s == b->own && s) { /* order after work the caller queued on the legacy default stream */
        cudaEvent_t ev;
        GCG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, 0);
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    const size_t cstride = ((size_t)nv + 63) & ~(size_t)63;
    const uint32_t nreal = b->roff[ng];
    if (!b->c.get()) {
        GCG_TRY(b->c.alloc(2 * cstride));
        GCG_TRY(b->rnz.alloc((size_t)2 * std::max<uint32_t>(pl.nnz, 1)));
        GCG_TRY(b->r.alloc(nv));
        GCG_TRY(b->nzsum.alloc(std::max<uint32_t>(pl.nnz, 1)));
        GCG_TRY(b->parts.alloc((size_t)2 * pl.nchunks + 2));
        GCG_TRY(b->tile_part.alloc(std::max<uint32_t>(b->ntiles, 1)));
        GCG_TRY(b->norm_const.alloc(ng));
        GCG_TRY(b->gres.alloc(ng));
        GCG_TRY(b->active.alloc(ng));
        GCG_TRY(b->gsweeps.alloc(ng));
        GCG_TRY(b->err.alloc(1));
        GCG_TRY(b->qctr.alloc(4));
        GCG_TRY(b->bar.alloc(2));
        GCG_TRY(b->rout.alloc(std::max<uint32_t>(nreal, 1)));
    }
    MultiArgs m;
    SweepArgs &a = m.a;
    memset(&m, 0, sizeof(m));
    a.col = pl.col_r.get();
    a.outdeg = u->outdeg.get();
    a.heads = (const uint8_t *)pl.head_bits.get();
    a.chunk_nz = pl.chunk_nz.get();
    a.nz_rows = pl.nz_rows.get();
    a.zero_rows = pl.zero_rows.get();
    a.split = pl.split.get();
    a.ne = u->ne;
    a.nchunks = pl.nchunks;
    a.nnz = pl.nnz;
    a.nzero = pl.nzero;
    a.nsplit = pl.nsplit;
    a.hub = std::min(pl.hub, b->tune_hub);
    a.nz_cidx = pl.nz_cidx.get();
    a.zero_cidx = pl.zero_cidx.get();
    a.od_nz = pl.od_nz.get();
    a.r_init = b->r.get();
    a.nzsum = b->nzsum.get();
    a.head_part = b->parts.get();
    a.tail_part = b->parts.get() + pl.nchunks + 1;
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.tol = p->tol;
    a.source = GCG_NO_SOURCE;
    m.c[0] = b->c.get();
    m.c[1] = b->c.get() + cstride;
    m.rnz[0] = b->rnz.get();
    m.rnz[1] = b->rnz.get() + pl.nnz;
    m.gr = b->gr.get();
    m.ng = ng;
    m.max_sweeps = (uint32_t)p->max_sweeps;
    m.tile_part = b->tile_part.get();
    m.norm_const = b->norm_const.get();
    m.active = b->active.get();
    m.gsweeps = b->gsweeps.get();
    m.gres = b->gres.get();
    m.qctr = b->qctr.get();
    m.bar = b->bar.get();
    m.err = b->err.get();
    const bool test_timeout = (p->flags & GCG_PR_TEST_BARRIER_TIMEOUT) != 0;
    m.spin_limit = test_timeout ? (1ll << 14) : (1ll << 25);
    m.extra_arrivals = test_timeout ? 1u : 0u;
    m.grab = b->tune_grab;
    m.voff = pl.per_interval ? b->d_voff.get() : nullptr;
    m.a.long_split = pl.long_split.get();
    m.long_g = b->long_g.get();
    m.nlong = pl.nlong;

    /* one cooperative launch: one CTA per SM, all resident; per-graph hubs may
     * start up to 3 entries before a graph's first id (16-byte alignment) */
    const uint32_t hub_bytes = (a.hub + (m.voff && a.hub ? 4u : 0u)) * 4u;
    GCG_CUDA(cudaFuncSetAttribute(k_multi_pagerank<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((HUB_MAX + 4) * 4)));
    GCG_CUDA(cudaFuncSetAttribute(k_multi_pagerank<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((HUB_MAX + 4) * 4)));
    int per_sm = 0;
    GCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, m.voff ? k_multi_pagerank<true> : k_multi_pagerank<false>, EDGE_THREADS, hub_bytes));
    if (per_sm < 1) return fail(GCG_ERR_UNSUPPORTED, "gcg_batch_pagerank: persistent kernel does not fit an SM");
    const unsigned grid = (unsigned)num_sms();

    /* initial vector given: caller layout (no padding) -> union layout, padding 0 */
    tbuf<float> init_stage, init_union;
    const float *init_dev = nullptr;
    if (p->init_rank) {
        const float *src = p->init_rank;
        if (!is_device_ptr(p->init_rank)) {
            GCG_TRY(init_stage.alloc(nreal, s));
            GCG_TRY(copy_in(init_stage.get(), p->init_rank, (size_t)nreal * 4, s));
            src = init_stage.get();
        }
        GCG_TRY(init_union.alloc(nv, s));
        GCG_CUDA(cudaMemsetAsync(init_union.get(), 0, (size_t)nv * 4, s));
        const dim3 eg((unsigned)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)nreal / ng + 255) / 256, 64)),
                      std::min<uint32_t>(ng, 1024));
        k_expand<<<eg, 256, 0, s>>>(src, b->d_roff.get(), b->d_voff.get(), ng, init_union.get(), 1);
        init_dev = init_union.get();
    }

    /* the whole solve as a CUDA graph, captured once per parameter set */
    bool use_graph = allow_graph && !p->init_rank && !test_timeout && !b->graph_unsupported;
    if (use_graph) {
        const bool same = b->gexec && b->key_t == p->teleport && b->key_d == p->damping && b->key_tol == p->tol &&
                          b->key_ms == p->max_sweeps && b->key_init == p->init && b->key_hub == a.hub &&
                          b->key_grab == m.grab;
        if (!same) {
            if (b->gexec) cudaGraphExecDestroy(b->gexec);
            b->gexec = nullptr;
            cudaGraph_t graph = nullptr;
            int rc = GCG_OK;
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                rc = GCG_ERR_CUDA;
            } else {
                rc = enqueue_solve(b, m, p, nullptr, grid, hub_bytes);
                if (cudaStreamEndCapture(s, &graph) != cudaSuccess) rc = GCG_ERR_CUDA;
            }
            if (rc == GCG_OK && cudaGraphInstantiate(&b->gexec, graph, 0) != cudaSuccess) rc = GCG_ERR_CUDA;
            if (graph) cudaGraphDestroy(graph);
            if (rc != GCG_OK) { /* this runtime cannot capture the solve: launch it directly from now on */
                cudaGetLastError();
                if (b->gexec) cudaGraphExecDestroy(b->gexec);
                b->gexec = nullptr;
                b->graph_unsupported = true;
                use_graph = false;
            } else {
                b->key_t = p->teleport;
                b->key_d = p->damping;
                b->key_tol = p->tol;
                b->key_ms = p->max_sweeps;
                b->key_init = p->init;
                b->key_hub = a.hub;
                b->key_grab = m.grab;
            }
        }
    }
    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    int rc = GCG_OK;
    if (use_graph) {
        cudaError_t e = cudaGraphLaunch(b->gexec, s);
        if (e != cudaSuccess) rc = fail(GCG_ERR_CUDA, std::string("gcg_batch_pagerank: graph launch: ") + cudaGetErrorString(e));
    } else {
        rc = enqueue_solve(b, m, p, init_dev, grid, hub_bytes);
    }
    cudaEventRecord(ev1, s);
    int herr = 0;
    std::vector<int> hsw(ng);
    std::vector<double> hres(ng);
    if (rc == GCG_OK) {
        cudaMemcpyAsync(&herr, b->err.get(), 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hsw.data(), b->gsweeps.get(), ng * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hres.data(), b->gres.get(), ng * 8, cudaMemcpyDeviceToHost, s);
    }
    cudaError_t se = cudaStreamSynchronize(s);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (rc != GCG_OK) return rc;
    if (se != cudaSuccess) return fail(GCG_ERR_CUDA, std::string("gcg_batch_pagerank: ") + cudaGetErrorString(se));
    if (herr) return fail(GCG_ERR_TIMEOUT, "gcg_batch_pagerank: a grid-barrier wait ran out (persistent kernel stopped)");
    if (out) GCG_TRY(copy_out(out, b->rout.get(), (size_t)nreal * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (sweeps) memcpy(sweeps, hsw.data(), ng * 4);
    if (residuals) memcpy(residuals, hres.data(), ng * 8);
    if (stats) {
        int mx = 0, conv = 1;
        double worst = 0.0;
        for (uint32_t g = 0; g < ng; ++g) {
            mx = std::max(mx, hsw[g]);
            worst = std::max(worst, hres[g]);
            if (!(p->tol > 0.0 && hres[g] <= p->tol)) conv = 0;
        }
        stats->sweeps = mx;
        stats->converged = conv;
        stats->residual = worst;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = ms;
        stats->timed_sweeps = mx;
        /* per-graph init, initial vector (2), the persistent kernel, the rank
         * assembly, the map to the callers' layout, and the map of init_rank */
        stats->kernel_launches = 6 + (p->init_rank ? 1 : 0);
        stats->levels = 0;
    }
    return GCG_OK;
}

/* Times `sweeps` fixed sweeps of every candidate launch configuration and keeps
 * the fastest: hub entries (the out-degree rank below which a source's
 * contribution is read from shared memory: the degree bin of the cache) and the
 * edge phase's work distribution (strided, or runs of 1, 4 or 16 chunks from
 * the device queue). */
static int batch_autotune(gcg_batch *b, int sweeps, uint32_t *hub_out, uint32_t *grab_out, double *ms_out) {
    const ChunkPlan &pl = *b->u->cplan;
    std::vector<uint32_t> hubs;
    for (uint32_t h : {0u, 8192u, 16384u, 32768u, HUB_DEFAULT, HUB_MAX})
        if (h <= pl.hub && std::find(hubs.begin(), hubs.end(), h) == hubs.end()) hubs.push_back(h);
    if (std::find(hubs.begin(), hubs.end(), pl.hub) == hubs.end()) hubs.push_back(pl.hub);
    /* with per-graph hubs the edge phase partitions the chunks statically: the
     * queue-run choice applies only to the one-hub layout */
    const std::vector<uint32_t> grabs = pl.per_interval ? std::vector<uint32_t>{0u}
                                                        : std::vector<uint32_t>{0u, 1u, 4u, 16u};
    gcg_pr_params p;
    gcg_pr_params_default(&p);
    p.max_sweeps = sweeps;
    p.tol = 0.0;
    double best = 1e300;
    uint32_t bh = pl.hub, bg = 0;
    for (uint32_t h : hubs)
        for (uint32_t g : grabs) {
            b->tune_hub = h;
            b->tune_grab = g;
            gcg_pr_stats st;
            double t = 1e300;
            for (int rep = 0; rep < 2; ++rep) { /* the first run warms caches and the pool */
                GCG_TRY(batch_pagerank(b, &p, nullptr, nullptr, nullptr, &st, false));
                t = std::min(t, st.device_ms);
            }
            if (t < best) {
                best = t;
                bh = h;
                bg = g;
            }
        }
    b->tune_hub = bh;
    b->tune_grab = bg;
    if (b->gexec) { /* captured with another configuration */
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
    }
    if (hub_out) *hub_out = bh;
    if (grab_out) *grab_out = bg;
    if (ms_out) *ms_out = best / std::max(sweeps, 1);
    return GCG_OK;
}

}  // namespace gcg

using namespace gcg;

extern "C" {

int gcg_batch_create(gcg_graph *const *graphs, uint32_t ngraphs, gcg_batch **out) {
    return gcg_batch_create_ex(graphs, ngraphs, 0u, out);
}

int gcg_batch_create_ex(gcg_graph *const *graphs, uint32_t ngraphs, uint32_t flags, gcg_batch **out) {
    if (!graphs || !out) return fail(GCG_ERR_INVALID, "gcg_batch_create: null argument");
    if (flags & ~GCG_BATCH_ONE_HUB) return fail(GCG_ERR_INVALID, "gcg_batch_create_ex: unknown flags");
    *out = nullptr;
    if (ngraphs == 0 || ngraphs > NG_MAX)
        return fail(GCG_ERR_INVALID, "gcg_batch_create: ngraphs must be 1.." + std::to_string(NG_MAX));
    for (uint32_t g = 0; g < ngraphs; ++g)
        if (!graphs[g]) return fail(GCG_ERR_INVALID, "gcg_batch_create: null graph");
    gcg_batch *b = new gcg_batch();
    int st = batch_build(graphs, ngraphs, flags, b);
    if (st == GCG_OK && cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) {
        b->own = nullptr;
        st = fail(GCG_ERR_CUDA, "gcg_batch_create: cannot create a stream");
    }
    if (st != GCG_OK) {
        delete b;
        return st;
    }
    b->u->stream = b->own;
    *out = b;
    return GCG_OK;
}

int gcg_batch_set_config(gcg_batch *b, uint32_t hub_entries, uint32_t queue_run) {
    if (!b) return fail(GCG_ERR_INVALID, "gcg_batch_set_config: null batch");
    if (queue_run > (1u << 20)) return fail(GCG_ERR_INVALID, "gcg_batch_set_config: queue_run too large");
    b->tune_hub = hub_entries;
    b->tune_grab = queue_run;
    return GCG_OK;
}

int gcg_batch_get_config(const gcg_batch *b, uint32_t *hub_entries, uint32_t *queue_run, int *graph_ready) {
    if (!b) return fail(GCG_ERR_INVALID, "gcg_batch_get_config: null batch");
    if (hub_entries) *hub_entries = std::min(b->u->cplan->hub, b->tune_hub);
    if (queue_run) *queue_run = b->tune_grab;
    if (graph_ready) *graph_ready = b->gexec != nullptr;
    return GCG_OK;
}

int gcg_batch_vertex_offsets(const gcg_batch *b, uint64_t *offsets) {
    if (!b || !offsets) return fail(GCG_ERR_INVALID, "gcg_batch_vertex_offsets: null argument");
    for (uint32_t g = 0; g <= b->ng; ++g) offsets[g] = b->roff[g];
    return GCG_OK;
}

int gcg_batch_set_stream(gcg_batch *b, void *stream) {
    if (!b) return fail(GCG_ERR_INVALID, "gcg_batch_set_stream: null batch");
    b->u->stream = stream ? (cudaStream_t)stream : b->own;
    return GCG_OK;
}

int gcg_batch_pagerank(gcg_batch *b, const gcg_pr_params *params, float *out_ranks, int32_t *sweeps,
                       double *residuals, gcg_pr_stats *stats) {
    if (!b || !params) return fail(GCG_ERR_INVALID, "gcg_batch_pagerank: null argument");
    if (params->mode != GCG_PR_JACOBI || params->source != GCG_NO_SOURCE)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_batch_pagerank: plain Jacobi only");
    if (params->max_sweeps < 0) return fail(GCG_ERR_INVALID, "gcg_batch_pagerank: max_sweeps < 0");
    return batch_pagerank(b, params, out_ranks, sweeps, residuals, stats);
}

int gcg_batch_autotune(gcg_batch *b, int sweeps, uint32_t *hub_entries, uint32_t *queue_run, double *ms_per_sweep) {
    if (!b) return fail(GCG_ERR_INVALID, "gcg_batch_autotune: null batch");
    if (sweeps < 1) return fail(GCG_ERR_INVALID, "gcg_batch_autotune: sweeps must be >= 1");
    return batch_autotune(b, sweeps, hub_entries, queue_run, ms_per_sweep);
}

int gcg_batch_free(gcg_batch *b) {
    if (!b) return GCG_OK;
    cudaStreamSynchronize(b->u ? b->u->stream : 0);
    delete b;
    return GCG_OK;
}

}  // extern "C"
