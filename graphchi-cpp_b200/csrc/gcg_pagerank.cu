/*
 * PageRank on the HBM-resident in-edge CSR (Jacobi / bulk-synchronous form).
 *
 * Replaces graphchi_engine::run() driving the PageRank update()
 * (src/engine/graphchi_engine.hpp:718-992; example_apps/pagerank.cpp:73-144;
 * example_apps/pagerank_functional.cpp:48-83 with
 * src/api/functional/functional_bulksync.hpp:91-113).
 *
 * One sweep = three kernels, all on the graph's stream:
 *   k_pr_edges   one warp per chunk of 256 consecutive in-edges (8 per lane):
 *                two 128-bit column loads per lane (streamed: no L1 allocation,
 *                L2 evict-first), eight independent gathers of contrib[src]
 *                (L2 evict-last, so the contrib vector stays resident while the
 *                columns stream past), row starts read from a 1-bit-per-edge
 *                head bitmap, in-lane segment sums, and a warp segmented scan
 *                (shuffles) to join rows across lanes. Rows inside the chunk get
 *                their sum written; a row crossing chunk boundaries leaves one
 *                partial per chunk.
 *   k_pr_fix     rows that cross chunks: partials added in chunk order.
 *   k_pr_vertex  apply for every vertex with in-edges:
 *                r' = (float)(teleport + damping*(double)sum), c' = r'/outdeg
 *                (float), FP64 |r'-r| and |r'|; the last block to finish reduces
 *                the block partials in a fixed order, logs the residual and raises
 *                `done` when it is <= tol (later queued sweeps return at once).
 *                Vertices without in-edges are constant (r' = teleport) and are
 *                written only in the first two sweeps (one per buffer).
 * Every sum is formed in a fixed order, so results are deterministic.
 * Algorithmic traffic per sweep: 8*E + 16*V bytes.
 */
#include <math.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"
#include "gcg_pr_device.cuh"

namespace gcg {

namespace {


/* ---- per-graph plan kernels -------------------------------------------- */
/* row_of[newid[v]] = v: the vertex at each position of the relabelled order */
__global__ void k_invert(const uint32_t *__restrict__ newid, uint32_t nv, uint32_t *__restrict__ row_of) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) row_of[newid[v]] = v;
}

/* in-degree of the row at each position j of the plan order (row_of[j], or j
 * when row_of is null) and whether it has in-edges */
__global__ void k_order_deg(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ row_of, uint32_t nv,
                            uint32_t *__restrict__ nzf, uint32_t *__restrict__ deg) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += gridDim.x * blockDim.x) {
        const uint32_t v = row_of ? row_of[j] : j;
        const uint32_t d = rowptr[v + 1] - rowptr[v];
        nzf[j] = d ? 1u : 0u;
        deg[j] = d;
    }
}

/* nz and zero rows in plan order; an nz row's edges start at the scanned
 * degree of its position (start[]) */
__global__ void k_split_rows(const uint32_t *__restrict__ row_of, const uint32_t *__restrict__ nzf, uint32_t nv,
                             const uint32_t *__restrict__ pos, const uint32_t *__restrict__ start,
                             uint32_t *__restrict__ nz_rows, uint32_t *__restrict__ nz_start,
                             uint32_t *__restrict__ zero_rows) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += gridDim.x * blockDim.x) {
        const uint32_t v = row_of ? row_of[j] : j;
        if (nzf[j]) {
            nz_rows[pos[j]] = v;
            nz_start[pos[j]] = start[j];
        } else {
            zero_rows[j - pos[j]] = v;
        }
    }
}

__global__ void k_head_bits(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint32_t *__restrict__ bits) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        uint32_t p = nz_start[i];
        atomicOr(bits + (p >> 5), 1u << (p & 31u));
    }
}

/* chunk_nz[c] = index of the non-empty row holding edge c*CH */
__global__ void k_chunk_nz(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint32_t nchunks,
                           uint32_t *__restrict__ chunk_nz) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        const uint64_t pos = (uint64_t)c * CH;
        uint32_t lo = 0, hi = nnz; /* largest i with nz_start[i] <= pos */
        while (hi - lo > 1) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if ((uint64_t)nz_start[mid] <= pos) lo = mid; else hi = mid;
        }
        chunk_nz[c] = lo;
    }
}

__global__ void k_split_flags(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint64_t ne,
                              uint32_t *__restrict__ f) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        uint64_t b = nz_start[i], e = (i + 1 < nnz) ? nz_start[i + 1] : ne;
        f[i] = ((b / CH) != ((e - 1) / CH)) ? 1u : 0u;
    }
}

__global__ void k_split_list(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint64_t ne,
                             const uint32_t *__restrict__ pos, uint4 *__restrict__ split) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        uint64_t b = nz_start[i], e = (i + 1 < nnz) ? nz_start[i + 1] : ne;
        uint32_t cs = (uint32_t)(b / CH), ce = (uint32_t)((e - 1) / CH);
        if (cs != ce) split[pos[i]] = make_uint4(i, cs, ce, 0u);
    }
}




/* Programmatic dependent launch: the three sweep kernels are queued with
 * programmatic stream serialisation, so a kernel's blocks may be scheduled while
 * its predecessor drains. Each kernel first waits (griddepcontrol.wait) until its
 * predecessor has completed and its writes are visible, and lets its own
 * successor be scheduled as soon as all its blocks are running. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

/* TEX: the gathers that miss the hub go through the texture path (a texture
 * object over c_old) instead of plain loads. The edge kernel is bound by the
 * L1TEX tag stage on these scattered gathers; at R-MAT scale 24 texture fetches
 * finish a launch ~6 % sooner than the same gathers as loads (same values). */
template <bool TEX>
__global__ void __launch_bounds__(EDGE_THREADS, 1) k_pr_edges(SweepArgs a) {
    pdl_wait();
    pdl_launch_next();
    if (*(volatile const int *)a.done) return;
    extern __shared__ __align__(16) float s_hub[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_fail;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();
    /* hub cache: contribs of the highest out-degree sources (relabelled
     * 0..hub-1), staged by one bulk copy (TMA) of its whole 16-byte part (c_old
     * and the hub are 16-byte aligned) while the warps load their first chunk;
     * the last hub % 4 entries by plain loads */
    const uint32_t hub4 = a.hub & ~3u;
    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(&s_bar, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0 && hub4) {
        mbar_arrive_expect_tx(&s_bar, hub4 * 4u);
        bulk_copy_g2s(s_hub, a.c_old, hub4 * 4u, &s_bar);
    }
    for (uint32_t i = hub4 + threadIdx.x; i < a.hub; i += blockDim.x) s_hub[i] = __ldcg(a.c_old + i);

    /* Warp w takes runs of a.run consecutive chunks: runs w, w + nwarps, ...
     * Software pipeline: while a chunk's gathers are in flight, the next chunk's
     * columns, head flags and row base are already being loaded. */
    const uint64_t R = a.run, nch = a.nchunks;
    uint64_t q = gwarp, ch = q * R, end = ch + R < nch ? ch + R : nch;
    uint32_t col[EPL], flags = 0, nvalid = 0, base = 0;
    if (ch < end) load_chunk(a, (uint32_t)ch, lane, pol_stream, col, flags, nvalid, base, a.ne);
    if (hub4) { /* bounded wait for the hub copy */
        bool ok = false;
        for (long long spin = 0; !ok && spin < MBAR_SPIN; ++spin) ok = mbar_try_wait(&s_bar, 0u);
        if (!ok) s_fail = 1;
    }
    __syncthreads(); /* also publishes the plainly loaded hub entries */
    if (s_fail) { /* the copy did not complete: report it and stop the solve */
        if (threadIdx.x == 0) {
            atomicExch(a.err, 1);
            atomicExch(a.done, 1);
        }
        return;
    }
    while (ch < end) {
        float val[EPL];
        if (TEX) {
#pragma unroll
            for (int j = 0; j < EPL; ++j) {
                const uint32_t x = col[j];
                float v = 0.0f;
                if ((uint32_t)j < nvalid) v = x < a.hub ? s_hub[x] : tex1Dfetch<float>(a.tex_old, (int)x);
                val[j] = v;
            }
        } else {
            gather_chunk(a, col, nvalid, s_hub, pol_keep, val);
        }
        const uint32_t cur = (uint32_t)ch, cur_flags = flags, cur_nvalid = nvalid, cur_base = base;
        if (++ch >= end) {
            q += nwarps;
            ch = q * R;
            end = ch + R < nch ? ch + R : nch;
        }
        if (ch < end) load_chunk(a, (uint32_t)ch, lane, pol_stream, col, flags, nvalid, base, a.ne);
        reduce_chunk(a, cur, lane, val, cur_flags, cur_nvalid, cur_base, a.ne);
    }
}

/* Rows that cross chunk boundaries: tail partial of the first chunk plus the
 * head partials of the later chunks. A warp takes 32 consecutive split rows;
 * each lane finishes its own row when it spans few chunks, and the warp sums the
 * partials of each long (hub) row cooperatively: lane-strided partial sums, then
 * a fixed xor-shuffle tree, so the order is fixed. */
/* Blocks [0, nlb) take the long rows, one warp per row (the fixed long-row
 * order: LONG_GROUPS lane-strided groups, each reduced by an xor tree, added in
 * group order); the other blocks take the short rows, one per lane, in chunk
 * order. */
constexpr uint32_t FIX_WARPS = 8; /* 256-thread blocks */
__global__ void __launch_bounds__(256) k_pr_fix(SweepArgs a) {
    pdl_wait();
    pdl_launch_next();
    if (*(volatile const int *)a.done) return;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nlb = (a.nlong + FIX_WARPS - 1) / FIX_WARPS;
    if (blockIdx.x < nlb) {
        const uint32_t r = blockIdx.x * FIX_WARPS + warp;
        if (r < a.nlong) {
            const uint4 sp = a.split[a.long_split[r]];
            const float t = long_row_sum_warp<false>(a.head_part, sp.y, sp.z, lane);
            if (lane == 0) a.nzsum[sp.x] = a.tail_part[sp.y] + t;
        }
        return;
    }
    const uint32_t nwarps = ((gridDim.x - nlb) * blockDim.x) >> 5;
    for (uint32_t wb = (((blockIdx.x - nlb) * blockDim.x + threadIdx.x) >> 5) * 32u; wb < a.nsplit;
         wb += nwarps * 32u) {
        const uint32_t k = wb + lane;
        if (k < a.nsplit) {
            const uint4 sp = a.split[k];
            if (sp.z - sp.y <= LONG_SPAN) {
                float s = a.tail_part[sp.y];
                for (uint32_t c = sp.y + 1; c <= sp.z; ++c) s += a.head_part[c];
                a.nzsum[sp.x] = s;
            }
        }
    }
}

/* personalised: the teleport term only at the source vertex */
__device__ __forceinline__ float pr_value_at(const SweepArgs &a, float sum, uint32_t v) {
    const double tele = (a.source == GCG_NO_SOURCE || v == a.source) ? a.teleport : 0.0;
    return (float)__dadd_rn(tele, __dmul_rn(a.damping, (double)sum));
}

__device__ __forceinline__ double2 block_sum2(double x, double y, double2 *s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        y += __shfl_down_sync(0xFFFFFFFFu, y, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_red[warp] = make_double2(x, y);
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            r.x += s_red[w].x;
            r.y += s_red[w].y;
        }
    __syncthreads();
    return r; /* valid in thread 0 */
}

__global__ void __launch_bounds__(256) k_pr_vertex(SweepArgs a, int sweep, int const_pass) {
    pdl_wait();
    pdl_launch_next();
    if (*(volatile const int *)a.done) return;
    __shared__ double2 s_red[8];
    __shared__ int s_last;
    double dsum = 0.0, nsum = 0.0;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    /* four rows (i, i + nth, i + 2 nth, i + 3 nth) per trip: their loads are all
     * issued before the first store; the residual sums keep the row order */
    constexpr int VB = 4;
    for (uint32_t i0 = tid; i0 < a.nnz; i0 += VB * nth) {
        float sum[VB], ro[VB];
        uint32_t od[VB], cid[VB], row[VB];
#pragma unroll
        for (int u = 0; u < VB; ++u) {
            const uint64_t i = (uint64_t)i0 + (uint64_t)u * nth;
            if (i < a.nnz) {
                if (a.ntiers > 1) { /* the row's tier partial sums, in tier order */
                    float t = 0.0f;
#pragma unroll
                    for (int k = 0; k < MAX_TIERS; ++k) {
                        if (k < (int)a.ntiers) {
                            const uint32_t j = a.tier_idx[(uint64_t)k * a.nnz + i];
                            if (j != GCG_NO_SOURCE) t += a.tier_sum[k][j];
                        }
                    }
                    sum[u] = t;
                } else {
                    sum[u] = a.nzsum[i];
                }
                ro[u] = a.r_nz_old[i];
                od[u] = a.od_nz[i];
                cid[u] = a.nz_cidx[i];
                row[u] = a.source == GCG_NO_SOURCE ? 0u : a.nz_rows[i];
            }
        }
#pragma unroll
        for (int u = 0; u < VB; ++u) {
            const uint64_t i = (uint64_t)i0 + (uint64_t)u * nth;
            if (i < a.nnz) {
                const float rn = a.source == GCG_NO_SOURCE ? pr_value(a, sum[u]) : pr_value_at(a, sum[u], row[u]);
                a.r_nz_new[i] = rn;
                a.c_new[cid[u]] = od[u] ? __fdiv_rn(rn, (float)od[u]) : 0.0f;
                dsum += fabs((double)rn - (double)ro[u]);
                nsum += fabs((double)rn);
            }
        }
    }
    if (const_pass) {
        /* vertices without in-edges: value teleport from the first sweep on;
         * written once into each contrib buffer (sweeps 0 and 1) */
        for (uint32_t i = tid; i < a.nzero; i += nth) {
            const uint32_t v = a.zero_rows[i];
            const float rn = pr_value_at(a, 0.0f, v);
            const float ro = sweep == 0 ? a.r_init[v] : rn;
            const uint32_t od = a.outdeg[v];
            a.c_new[a.zero_cidx[i]] = od ? __fdiv_rn(rn, (float)od) : 0.0f;
            dsum += fabs((double)rn - (double)ro);
            nsum += fabs((double)rn);
        }
    }
    double2 r = block_sum2(dsum, nsum, s_red);
    if (threadIdx.x == 0) {
        a.block_res[blockIdx.x] = r;
        __threadfence();
        s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double x = 0.0, y = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        double2 p = __ldcg(a.block_res + i);
        x += p.x;
        y += p.y;
    }
    double2 tot = block_sum2(x, y, s_red);
    if (threadIdx.x == 0) {
        const double norm = tot.y + (const_pass ? 0.0 : a.norm_const);
        const double res = norm > 0.0 ? tot.x / norm : 0.0;
        a.res_log[sweep] = res;
        if (a.delta_log) a.delta_log[sweep] = tot.x;
        *a.last_res = res;
        *a.sweeps_done = sweep + 1;
        if (a.tol > 0.0 && res <= a.tol) *a.done = 1;
        *a.ticket = 0u;
    }
}

/* r = initial vector (original ids); c = contribs at relabelled ids */
__global__ void k_pr_init(uint32_t nv, const uint32_t *__restrict__ outdeg, const uint32_t *__restrict__ newid,
                          float init, const float *__restrict__ init_rank, uint32_t source, float *__restrict__ r,
                          float *__restrict__ c) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        /* personalised runs start from the indicator of the source */
        float x = init_rank ? init_rank[v] : (source == GCG_NO_SOURCE ? init : (v == source ? 1.0f : 0.0f));
        r[v] = x;
        uint32_t od = outdeg[v];
        c[newid[v]] = od ? __fdiv_rn(x, (float)od) : 0.0f;
    }
}

/* relabelling by out-degree (descending, ties by id): keys sort ascending */
__global__ void k_outdeg_keys(const uint32_t *__restrict__ outdeg, uint32_t nv, uint32_t maxdeg, uint32_t vbits,
                              uint64_t *__restrict__ keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)(maxdeg - outdeg[v]) << vbits) | v;
}

/* the same keys led by the vertex's interval (last vertex ids ascending), so the
 * relabelling keeps every interval's id range */
__global__ void k_outdeg_keys_iv(const uint32_t *__restrict__ outdeg, uint32_t nv, uint32_t maxdeg, uint32_t vbits,
                                 uint32_t dbits, const uint32_t *__restrict__ last, uint32_t nint,
                                 uint64_t *__restrict__ keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nint - 1; /* first interval whose last vertex is >= v */
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (last[mid] < v) lo = mid + 1; else hi = mid;
        }
        keys[v] = ((uint64_t)lo << (dbits + vbits)) | ((uint64_t)(maxdeg - outdeg[v]) << vbits) | v;
    }
}

__global__ void k_newid(const uint64_t *__restrict__ sorted, uint32_t nv, uint32_t vbits, uint32_t *__restrict__ newid) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        newid[(uint32_t)(sorted[i] & mask)] = i;
}

/* col_r = newid[col] of the rows in plan order, in the chunk layout of
 * load_chunk (chunk_slot), whole chunks (slots past the last edge hold 0): one
 * warp per chunk. The rows overlapping the chunk are consecutive from
 * chunk_nz[c]; the warp reads their extents and CSR offsets 32 rows at a time
 * (one lane per row), then copies each row's piece with all lanes, each row's
 * sources in their CSR order. */
__global__ void k_relabel_rows(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col,
                               const uint32_t *__restrict__ nz_rows, const uint32_t *__restrict__ nz_start,
                               uint32_t nnz, uint64_t ne, uint32_t nchunks, const uint32_t *__restrict__ chunk_nz,
                               const uint32_t *__restrict__ newid, uint32_t *__restrict__ col_r) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = w0; c < nchunks; c += nw) {
        const uint64_t c0 = c * CH, c1 = c0 + CH < ne ? c0 + CH : ne;
        for (uint64_t e = c1 + lane; e < c0 + CH; e += 32) col_r[chunk_slot(e)] = 0u;
        for (uint32_t ib = chunk_nz[c];; ib += 32u) {
            const uint32_t i = ib + lane;
            uint64_t rs = 0, re = 0, src = 0;
            bool have = false;
            if (i < nnz) {
                rs = nz_start[i];
                if (rs < c1) {
                    have = true;
                    re = i + 1 < nnz ? nz_start[i + 1] : ne;
                    src = rowptr[nz_rows[i]];
                }
            }
            const uint32_t hm = __ballot_sync(0xFFFFFFFFu, have); /* a prefix of the lanes */
            for (uint32_t m = hm; m; m &= m - 1u) {
                const int j = __ffs((int)m) - 1;
                const uint64_t rsj = __shfl_sync(0xFFFFFFFFu, rs, j), rej = __shfl_sync(0xFFFFFFFFu, re, j);
                const uint64_t srcj = __shfl_sync(0xFFFFFFFFu, src, j);
                const uint64_t lo = rsj > c0 ? rsj : c0, hi = rej < c1 ? rej : c1;
                for (uint64_t e = lo + lane; e < hi; e += 32) col_r[chunk_slot(e)] = newid[col[srcj + (e - rsj)]];
            }
            if (hm != 0xFFFFFFFFu) break; /* the chunk's last row was in this batch */
        }
    }
}

__global__ void k_max_u32(const uint32_t *__restrict__ a, uint32_t n, uint32_t *out) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

/* compact state of the vertices with in-edges */
__global__ void k_pr_init_nz(uint32_t nnz, const uint32_t *__restrict__ nz_rows, const float *__restrict__ r,
                             float *__restrict__ r_nz) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x)
        r_nz[i] = r[nz_rows[i]];
}

/* assemble the full rank vector after the last sweep */
__global__ void k_pr_scatter(uint32_t nnz, uint32_t nzero, const uint32_t *__restrict__ nz_rows,
                             const uint32_t *__restrict__ zero_rows, const float *__restrict__ r_nz, float t,
                             uint32_t source, float *__restrict__ r) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < nnz; i += nth) r[nz_rows[i]] = r_nz[i];
    for (uint32_t i = tid; i < nzero; i += nth) {
        const uint32_t v = zero_rows[i];
        r[v] = (source == GCG_NO_SOURCE || v == source) ? t : 0.0f;
    }
}

__global__ void k_gather_u32(uint32_t n, const uint32_t *__restrict__ idx, const uint32_t *__restrict__ src,
                             uint32_t *__restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

__global__ void k_long_list(const uint4 *__restrict__ split, uint32_t nsplit, uint32_t *count,
                            uint32_t *__restrict__ list) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nsplit; i += gridDim.x * blockDim.x) {
        const uint4 sp = split[i];
        if (sp.z - sp.y > LONG_SPAN) list[atomicAdd(count, 1u)] = i;
    }
}

/* ---- source tiers ---------------------------------------------------------- */
/* tier of each edge: k >= 1 when its relabelled source lies in [k w, (k+1) w)
 * for k < ntiers, else 0 */
__global__ void k_edge_tier(const uint32_t *__restrict__ col_r, uint64_t ne, uint32_t width, uint32_t ntiers,
                            uint8_t *__restrict__ tier) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = col_r[chunk_slot(e)] / width;
        tier[e] = (uint8_t)(k < ntiers ? k : 0u);
    }
}

/* f[e] = (tier[e] == k) for e < ne, f[ne] = 0 (so the exclusive scan ends with the total) */
__global__ void k_tier_flags(const uint8_t *__restrict__ tier, uint64_t ne, uint8_t k, uint32_t *__restrict__ f) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e <= ne; e += (uint64_t)gridDim.x * blockDim.x)
        f[e] = e < ne && tier[e] == k ? 1u : 0u;
}

/* rows of tier k: nz row i (edges [nz_start[i], next start or ne) in plan
 * order) has tier-k edges when the scanned positions at its two ends differ */
__global__ void k_tier_row_flags(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint64_t ne,
                                 const uint32_t *__restrict__ epos, uint32_t *__restrict__ rf) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        const uint64_t e1 = i + 1 < nnz ? nz_start[i + 1] : ne;
        rf[i] = epos[e1] > epos[nz_start[i]] ? 1u : 0u;
    }
}

__global__ void k_tier_rows(const uint32_t *__restrict__ nz_start, uint32_t nnz, uint64_t ne,
                            const uint32_t *__restrict__ epos, const uint32_t *__restrict__ rpos,
                            uint32_t *__restrict__ idx, uint32_t *__restrict__ start) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
        const uint64_t e1 = i + 1 < nnz ? nz_start[i + 1] : ne;
        const uint32_t b = epos[nz_start[i]];
        if (epos[e1] > b) {
            idx[i] = rpos[i];
            start[rpos[i]] = b;
        } else {
            idx[i] = GCG_NO_SOURCE;
        }
    }
}

/* tier k's columns in the chunk layout, relative to the tier's first id */
__global__ void k_tier_cols(const uint32_t *__restrict__ col_r, uint64_t ne, const uint8_t *__restrict__ tier,
                            uint8_t k, uint32_t first, const uint32_t *__restrict__ epos,
                            uint32_t *__restrict__ out) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += (uint64_t)gridDim.x * blockDim.x)
        if (tier[e] == k) out[chunk_slot(epos[e])] = col_r[chunk_slot(e)] - first;
}

inline unsigned grid1d(uint64_t n, uint64_t cap_per_sm = 16) {
    uint64_t b = (n + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * cap_per_sm;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

/* ---- the chunk plan: built once per graph -------------------------------- */
void free_chunk_plan(ChunkPlan *p) { delete p; }

/* initial state of a sweep: full rank vector r, contributions c (relabelled,
 * buffer 0) and the compact ranks of the vertices with in-edges (buffer 0) */
int pr_init_state(gcg_graph *g, float init, const float *init_dev, float *r, float *c, float *rnz) {
    const ChunkPlan &pl = *g->cplan;
    cudaStream_t s = g->stream;
    k_pr_init<<<grid1d(g->nv, 8), 256, 0, s>>>(g->nv, g->outdeg.get(), pl.newid.get(), init, init_dev, GCG_NO_SOURCE,
                                               r, c);
    k_pr_init_nz<<<grid1d(pl.nnz, 8), 256, 0, s>>>(pl.nnz, pl.nz_rows.get(), r, rnz);
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

/* Row structure of an edge array grouped by row (nrows non-empty rows starting
 * at edge positions nz_start[], ne edges): the 1-bit-per-edge row-start bitmap,
 * each 256-edge chunk's starting row, the rows crossing chunk boundaries and,
 * among them, those spanning more than LONG_SPAN chunks. */
static int build_segments(const uint32_t *nz_start, uint32_t nrows, uint64_t ne, cudaStream_t s, uint32_t &nchunks,
                          dbuf<uint32_t> &head_bits, dbuf<uint32_t> &chunk_nz, dbuf<uint4> &split,
                          dbuf<uint32_t> &long_split, uint32_t &nsplit, uint32_t &nlong) {
    nchunks = (uint32_t)((ne + CH - 1) / CH);
    nsplit = nlong = 0;
    /* head bitmap covers whole chunks plus one spare word (read of the next chunk's first bit) */
    const uint64_t words = ((uint64_t)nchunks * CH) / 32 + 8;
    GCG_TRY(head_bits.alloc(words));
    GCG_TRY(chunk_nz.alloc(std::max<uint32_t>(nchunks, 1)));
    GCG_CUDA(cudaMemsetAsync(head_bits.get(), 0, words * 4, s));
    if (!nrows) return split.alloc(1);
    tbuf<uint32_t> flags, pos, total;
    GCG_TRY(flags.alloc(nrows, s));
    GCG_TRY(pos.alloc(nrows, s));
    GCG_TRY(total.alloc(1, s));
    k_head_bits<<<grid1d(nrows), 256, 0, s>>>(nz_start, nrows, head_bits.get());
    k_chunk_nz<<<grid1d(nchunks), 256, 0, s>>>(nz_start, nrows, nchunks, chunk_nz.get());
    k_split_flags<<<grid1d(nrows), 256, 0, s>>>(nz_start, nrows, ne, flags.get());
    GCG_TRY(scan_u32(flags.get(), pos.get(), nrows, total.get(), s));
    GCG_CUDA(cudaMemcpyAsync(&nsplit, total.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    GCG_TRY(split.alloc(std::max<uint32_t>(nsplit, 1)));
    k_split_list<<<grid1d(nrows), 256, 0, s>>>(nz_start, nrows, ne, pos.get(), split.get());
    /* the long split rows, each summed by a block of the fix-up (any order) */
    if (nsplit) {
        GCG_CUDA(cudaMemsetAsync(total.get(), 0, 4, s));
        GCG_TRY(long_split.alloc(nsplit));
        k_long_list<<<grid1d(nsplit), 256, 0, s>>>(split.get(), nsplit, total.get(), long_split.get());
        GCG_CUDA(cudaMemcpyAsync(&nlong, total.get(), 4, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
    }
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

int ensure_chunk_plan(gcg_graph *g) {
    if (g->cplan) return GCG_OK;
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv;
    const uint64_t ne = g->ne;
    ChunkPlan *p = new ChunkPlan();
    auto bail = [&](int st) {
        delete p;
        return st;
    };
    p->nchunks = (uint32_t)((ne + CH - 1) / CH);
    int st = GCG_OK;
    /* relabel sources by out-degree so the hottest contribs sit at ids [0, hub) */
    {
        tbuf<uint32_t> dmax;
        tbuf<uint64_t> keys, tmp;
        if (dmax.alloc(1, s) || keys.alloc(std::max<uint32_t>(nv, 1), s) || tmp.alloc(std::max<uint32_t>(nv, 1), s) ||
            p->newid.alloc(std::max<uint32_t>(nv, 1)))
            return bail(GCG_ERR_NOMEM);
        cudaMemsetAsync(dmax.get(), 0, 4, s);
        k_max_u32<<<grid1d(nv), 256, 0, s>>>(g->outdeg.get(), nv, dmax.get());
        uint32_t maxdeg = 0;
        if (cudaMemcpyAsync(&maxdeg, dmax.get(), 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return bail(fail(GCG_ERR_CUDA, "chunk plan: readback"));
        uint32_t dbits = 1;
        while (dbits < 32 && (1ull << dbits) <= maxdeg) ++dbits;
        uint32_t ibits = 1;
        while (ibits < 32 && (1ull << ibits) < g->nshards) ++ibits;
        p->per_interval = g->relabel_per_interval && g->nshards > 1 && g->intervals_dev.get() &&
                          g->vbits + dbits + ibits <= 64;
        uint64_t *sorted = nullptr;
        if (p->per_interval) {
            k_outdeg_keys_iv<<<grid1d(nv), 256, 0, s>>>(g->outdeg.get(), nv, maxdeg, g->vbits, dbits,
                                                        g->intervals_dev.get(), g->nshards, keys.get());
            if ((st = radix_sort_u64(keys.get(), tmp.get(), nv, (int)g->vbits, (int)(g->vbits + dbits + ibits),
                                     &sorted, s)))
                return bail(st);
        } else {
            k_outdeg_keys<<<grid1d(nv), 256, 0, s>>>(g->outdeg.get(), nv, maxdeg, g->vbits, keys.get());
            if ((st = radix_sort_u64(keys.get(), tmp.get(), nv, (int)g->vbits, (int)(g->vbits + dbits), &sorted, s)))
                return bail(st);
        }
        k_newid<<<grid1d(nv), 256, 0, s>>>(sorted, nv, g->vbits, p->newid.get());
        p->hub = std::min<uint32_t>(nv, HUB_MAX);
    }
    /* rows in relabelled order, unless this is a union whose relabelling mixes
     * its graphs' id ranges (each graph's rows must stay one contiguous range) */
    p->rows_relabelled = !g->union_of_graphs || p->per_interval;
    tbuf<uint32_t> row_of, nzf, pos, start, total;
    const uint64_t nv1 = std::max<uint64_t>(nv, 1);
    if (nzf.alloc(nv1, s) || pos.alloc(nv1, s) || start.alloc(nv1, s) || total.alloc(1, s) ||
        (p->rows_relabelled && row_of.alloc(nv1, s)))
        return bail(GCG_ERR_NOMEM);
    if (p->rows_relabelled) k_invert<<<grid1d(nv), 256, 0, s>>>(p->newid.get(), nv, row_of.get());
    k_order_deg<<<grid1d(nv), 256, 0, s>>>(g->in_rowptr.get(), p->rows_relabelled ? row_of.get() : nullptr, nv,
                                           nzf.get(), start.get());
    if ((st = scan_u32(nzf.get(), pos.get(), nv, total.get(), s))) return bail(st);
    uint32_t nnz = 0;
    if (cudaMemcpyAsync(&nnz, total.get(), 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return bail(fail(GCG_ERR_CUDA, "chunk plan: readback"));
    if ((st = scan_u32(start.get(), start.get(), nv, nullptr, s))) return bail(st);
    p->nnz = nnz;
    p->nzero = nv - nnz;
    if (p->nz_rows.alloc(std::max<uint32_t>(nnz, 1)) || p->nz_start.alloc(std::max<uint32_t>(nnz, 1)) ||
        p->zero_rows.alloc(std::max<uint32_t>(p->nzero, 1)) || p->od_nz.alloc(std::max<uint32_t>(nnz, 1)) ||
        p->nz_cidx.alloc(std::max<uint32_t>(nnz, 1)) || p->zero_cidx.alloc(std::max<uint32_t>(p->nzero, 1)) ||
        p->col_r.alloc(std::max<uint64_t>((uint64_t)p->nchunks * CH, CH)))
        return bail(GCG_ERR_NOMEM);
    k_split_rows<<<grid1d(nv), 256, 0, s>>>(p->rows_relabelled ? row_of.get() : nullptr, nzf.get(), nv, pos.get(),
                                            start.get(), p->nz_rows.get(), p->nz_start.get(), p->zero_rows.get());
    if (nnz) {
        k_gather_u32<<<grid1d(nnz), 256, 0, s>>>(nnz, p->nz_rows.get(), g->outdeg.get(), p->od_nz.get());
        k_gather_u32<<<grid1d(nnz), 256, 0, s>>>(nnz, p->nz_rows.get(), p->newid.get(), p->nz_cidx.get());
    }
    if (p->nzero)
        k_gather_u32<<<grid1d(p->nzero), 256, 0, s>>>(p->nzero, p->zero_rows.get(), p->newid.get(),
                                                     p->zero_cidx.get());
    if ((st = build_segments(p->nz_start.get(), nnz, ne, s, p->nchunks, p->head_bits, p->chunk_nz, p->split,
                             p->long_split, p->nsplit, p->nlong)))
        return bail(st);
    if (p->nchunks)
        k_relabel_rows<<<grid1d((uint64_t)p->nchunks * 32, 32), 256, 0, s>>>(
            g->in_rowptr.get(), g->in_col.get(), p->nz_rows.get(), p->nz_start.get(), nnz, ne, p->nchunks,
            p->chunk_nz.get(), p->newid.get(), p->col_r.get());
    else
        cudaMemsetAsync(p->col_r.get(), 0, CH * 4, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(GCG_ERR_CUDA, "chunk plan: relabel"));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bail(fail(GCG_ERR_CUDA, std::string("chunk plan: ") + cudaGetErrorString(e)));
    g->cplan = p;
    return GCG_OK;
}

int ensure_tier_plan(gcg_graph *g, int ntiers, uint32_t width) {
    GCG_TRY(ensure_chunk_plan(g));
    ChunkPlan &pl = *g->cplan;
    TierPlan &tp = pl.tiers;
    if (tp.ntiers == ntiers && tp.width == width) return GCG_OK;
    if (ntiers < 2 || ntiers > MAX_TIERS || width == 0 || (width & 3u))
        return fail(GCG_ERR_INVALID, "source tiers: 2..4 tiers of a width that is a multiple of 4");
    tp.ntiers = 0;
    cudaStream_t s = g->stream;
    const uint64_t ne = g->ne;
    const uint32_t nnz = pl.nnz;
    if (ne >= 0xFFFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "source tiers: too many edges");
    tbuf<uint8_t> tier;
    tbuf<uint32_t> epos, rflag, rpos, start, total;
    GCG_TRY(tier.alloc(std::max<uint64_t>(ne, 1), s));
    GCG_TRY(epos.alloc(ne + 1, s));
    GCG_TRY(rflag.alloc(std::max<uint32_t>(nnz, 1), s));
    GCG_TRY(rpos.alloc(std::max<uint32_t>(nnz, 1), s));
    GCG_TRY(start.alloc(std::max<uint32_t>(nnz, 1), s));
    GCG_TRY(total.alloc(1, s));
    GCG_TRY(tp.idx.alloc((size_t)ntiers * std::max<uint32_t>(nnz, 1)));
    if (ne)
        k_edge_tier<<<grid1d(ne, 32), 256, 0, s>>>(pl.col_r.get(), ne, width, (uint32_t)ntiers, tier.get());
    for (int k = 0; k < ntiers; ++k) {
        EdgeTier &t = tp.t[k];
        k_tier_flags<<<grid1d(ne + 1, 32), 256, 0, s>>>(tier.get(), ne, (uint8_t)k, epos.get());
        GCG_TRY(scan_u32(epos.get(), epos.get(), ne + 1, total.get(), s));
        uint32_t tne = 0;
        GCG_CUDA(cudaMemcpyAsync(&tne, total.get(), 4, cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
        t.ne = tne;
        t.first = k == 0 ? 0u : (uint32_t)k * width;
        t.hub = k == 0 ? std::min(width, g->nv)
                       : (t.first < g->nv ? std::min<uint32_t>(width, g->nv - t.first) : 0u); /* empty past nv */
        uint32_t nrows = 0;
        if (nnz) {
            k_tier_row_flags<<<grid1d(nnz), 256, 0, s>>>(pl.nz_start.get(), nnz, ne, epos.get(), rflag.get());
            GCG_TRY(scan_u32(rflag.get(), rpos.get(), nnz, total.get(), s));
            GCG_CUDA(cudaMemcpyAsync(&nrows, total.get(), 4, cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            k_tier_rows<<<grid1d(nnz), 256, 0, s>>>(pl.nz_start.get(), nnz, ne, epos.get(), rpos.get(),
                                                   tp.idx.get() + (size_t)k * nnz, start.get());
        }
        t.nrows = nrows;
        GCG_TRY(build_segments(start.get(), nrows, tne, s, t.nchunks, t.head_bits, t.chunk_nz, t.split, t.long_split,
                               t.nsplit, t.nlong));
        const uint64_t slots = std::max<uint64_t>((uint64_t)t.nchunks * CH, CH);
        GCG_TRY(t.col.alloc(slots));
        GCG_CUDA(cudaMemsetAsync(t.col.get(), 0, slots * 4, s));
        if (ne)
            k_tier_cols<<<grid1d(ne, 32), 256, 0, s>>>(pl.col_r.get(), ne, tier.get(), (uint8_t)k, t.first,
                                                       epos.get(), t.col.get());
        GCG_TRY(t.nzsum.alloc(std::max<uint32_t>(nrows, 1)));
        GCG_TRY(t.parts.alloc((size_t)2 * t.nchunks + 2));
        GCG_LAUNCH_CHECK();
    }
    GCG_CUDA(cudaStreamSynchronize(s));
    tp.ntiers = ntiers;
    tp.width = width;
    return GCG_OK;
}

/* queues kern<<<grid, block, smem, s>>>(args...) with programmatic stream
 * serialisation (the kernel must begin with pdl_wait) */
template <typename... K, typename... Args>
static void launch_pdl(void (*kern)(K...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

/* one CTA of EDGE_THREADS per SM (the hub cache takes most of shared memory) */
static void launch_edges(int ge, uint32_t hub_bytes, cudaStream_t s, const SweepArgs &a) {
    if (a.tex_old)
        launch_pdl(k_pr_edges<true>, ge, EDGE_THREADS, hub_bytes, s, a);
    else
        launch_pdl(k_pr_edges<false>, ge, EDGE_THREADS, hub_bytes, s, a);
}

static int edge_grid(uint32_t hub_bytes) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_pr_edges<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(HUB_MAX * 4));
        cudaFuncSetAttribute(k_pr_edges<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(HUB_MAX * 4));
        attr = true;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_edges<false>, EDGE_THREADS, hub_bytes) != cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = 1;
    }
    return num_sms() * per_sm;
}

static int pagerank_jacobi(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats) {
    GCG_TRY(ensure_chunk_plan(g));
    cudaStream_t s = g->stream;
    const ChunkPlan &pl = *g->cplan;
    const uint32_t nv = g->nv;
    const int max_sweeps = p->max_sweeps;

    const uint32_t hub_bytes = std::min(pl.hub, pl.tune_hub) * 4u;
    const uint64_t run = std::max(1u, pl.tune_run);
    const int ge = std::max(1, (int)std::min<uint64_t>((uint64_t)edge_grid(hub_bytes), (pl.nchunks + 32 * run - 1) / (32 * run)));
    const int gv = (int)grid1d(std::max<uint64_t>(pl.nnz, pl.nzero), 16);
    /* the sweep workspace lives with the graph: allocated on the first call,
     * reused by later calls (no allocation on the repeated-solve path) */
    PrWork &w = g->cplan->work;
    /* each contrib buffer starts on a 512-byte boundary (vector loads of the hub,
     * texture alignment) */
    const size_t cstride = ((size_t)nv + 127) & ~(size_t)127;
    if (!w.r.get()) {
        GCG_TRY(w.r.alloc((size_t)nv));
        GCG_TRY(w.rnz.alloc((size_t)2 * std::max<uint32_t>(pl.nnz, 1)));
        GCG_TRY(w.c.alloc((size_t)2 * cstride));
        GCG_TRY(w.nzsum.alloc(std::max<uint32_t>(pl.nnz, 1)));
        GCG_TRY(w.parts.alloc((size_t)2 * pl.nchunks + 2));
        GCG_TRY(w.bres.alloc(gv));
        GCG_TRY(w.ctl.alloc(4));
        GCG_CUDA(host_alloc((void **)&w.h_flags, 64 * sizeof(int)));
        for (int h = 0; h < 2; ++h) { /* no texture (too large, misaligned): plain loads */
            cudaResourceDesc rd = {};
            rd.resType = cudaResourceTypeLinear;
            rd.res.linear.devPtr = w.c.get() + (size_t)h * cstride;
            rd.res.linear.desc = cudaCreateChannelDesc<float>();
            rd.res.linear.sizeInBytes = (size_t)nv * 4;
            cudaTextureDesc td = {};
            td.readMode = cudaReadModeElementType;
            cudaTextureObject_t t = 0;
            if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
                cudaGetLastError();
                t = 0;
            }
            w.tex[h] = (unsigned long long)t;
        }
        if (!w.tex[0] || !w.tex[1]) {
            for (unsigned long long &t : w.tex) {
                if (t) cudaDestroyTextureObject((cudaTextureObject_t)t);
                t = 0;
            }
        }
    }
    if (w.dres.n < 2 * (size_t)max_sweeps + 1) GCG_TRY(w.dres.alloc(2 * (size_t)max_sweeps + 1));
    dbuf<float> &r = w.r, &c = w.c, &nzsum = w.nzsum, &parts = w.parts, &rnz = w.rnz;
    dbuf<double2> &bres = w.bres;
    dbuf<uint32_t> &ctl = w.ctl; /* ticket, done, sweeps_done */
    dbuf<double> &dres = w.dres; /* res_log[max_sweeps] + last_res */
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 4 * sizeof(uint32_t), s));
    GCG_CUDA(cudaMemsetAsync(dres.get(), 0, (2 * (size_t)max_sweeps + 1) * sizeof(double), s));

    /* initial vector: caller's (warm start) or the constant init */
    tbuf<float> init_stage;
    const float *init_dev = nullptr;
    if (p->init_rank) {
        if (is_device_ptr(p->init_rank)) {
            init_dev = p->init_rank;
        } else {
            GCG_TRY(init_stage.alloc(nv, s));
            GCG_TRY(copy_in(init_stage.get(), p->init_rank, (size_t)nv * 4, s));
            init_dev = init_stage.get();
        }
    }
    k_pr_init<<<grid1d(nv, 8), 256, 0, s>>>(nv, g->outdeg.get(), pl.newid.get(), p->init, init_dev, p->source, r.get(),
                                            c.get());
    k_pr_init_nz<<<grid1d(pl.nnz, 8), 256, 0, s>>>(pl.nnz, pl.nz_rows.get(), r.get(), rnz.get());
    GCG_LAUNCH_CHECK();

    SweepArgs a{};
    a.col = pl.col_r.get();
    a.hub = std::min(pl.hub, pl.tune_hub);
    a.run = std::max(1u, pl.tune_run);
    a.nz_cidx = pl.nz_cidx.get();
    a.zero_cidx = pl.zero_cidx.get();
    a.outdeg = g->outdeg.get();
    a.heads = (const uint8_t *)pl.head_bits.get();
    a.chunk_nz = pl.chunk_nz.get();
    a.nz_rows = pl.nz_rows.get();
    a.zero_rows = pl.zero_rows.get();
    a.split = pl.split.get();
    a.long_split = pl.long_split.get();
    a.nlong = pl.nlong;
    a.ne = g->ne;
    a.nchunks = pl.nchunks;
    a.nnz = pl.nnz;
    a.nzero = pl.nzero;
    a.nsplit = pl.nsplit;
    a.od_nz = pl.od_nz.get();
    a.r_init = r.get();
    a.nzsum = nzsum.get();
    a.head_part = parts.get();
    a.tail_part = parts.get() + pl.nchunks + 1;
    a.block_res = bres.get();
    a.ticket = ctl.get();
    a.done = (int *)(ctl.get() + 1);
    a.sweeps_done = (int *)(ctl.get() + 2);
    a.err = (int *)(ctl.get() + 3);
    a.res_log = dres.get();
    a.last_res = dres.get() + max_sweeps;
    a.delta_log = (p->delta_log || p->work_log) ? dres.get() + max_sweeps + 1 : nullptr;
    a.teleport = p->teleport;
    a.damping = p->damping;
    a.tol = p->tol;
    /* |r'| of the constant vertices, added to the norm once they are no longer visited */
    a.source = p->source;
    if (p->source == GCG_NO_SOURCE) {
        a.norm_const = (double)pl.nzero * fabs((double)(float)p->teleport);
    } else { /* only the source keeps a teleport value, if it has no in-edges */
        uint32_t sdeg = 0;
        GCG_CUDA(cudaMemcpy(&sdeg, g->indeg.get() + p->source, 4, cudaMemcpyDeviceToHost));
        a.norm_const = sdeg == 0 ? fabs((double)(float)p->teleport) : 0.0;
    }
    /* + a block per FIX_WARPS long rows */
    const int fg = (int)grid1d(std::max<uint32_t>(pl.nsplit, 1), 32) + (int)((pl.nlong + FIX_WARPS - 1) / FIX_WARPS);

    /* source tiers: one edge pass per tier, each with its tier's contributions in
     * shared memory (tier 0: the hub plus every source past the last tier) */
    const uint32_t tier_width = (hub_bytes / 4u) & ~3u; /* a multiple of 4: tier hubs load as float4 */
    const int ntiers =
        (pl.tune_tiers > 1 && tier_width > 0) ? (int)std::min<uint32_t>(pl.tune_tiers, MAX_TIERS) : 1;
    SweepArgs at[MAX_TIERS];
    int ge_t[MAX_TIERS], fg_t[MAX_TIERS];
    if (ntiers > 1) {
        GCG_TRY(ensure_tier_plan(g, ntiers, tier_width));
        const TierPlan &tp = g->cplan->tiers;
        a.ntiers = (uint32_t)ntiers;
        a.tier_idx = tp.idx.get();
        for (int k = 0; k < ntiers; ++k) {
            const EdgeTier &t = tp.t[k];
            SweepArgs &b = at[k];
            b = a;
            b.col = t.col.get();
            b.heads = (const uint8_t *)t.head_bits.get();
            b.chunk_nz = t.chunk_nz.get();
            b.split = t.split.get();
            b.long_split = t.long_split.get();
            b.nlong = t.nlong;
            b.nsplit = t.nsplit;
            b.nchunks = t.nchunks;
            b.ne = t.ne;
            b.hub = t.hub;
            b.nzsum = t.nzsum.get();
            b.head_part = t.parts.get();
            b.tail_part = t.parts.get() + t.nchunks + 1;
            a.tier_sum[k] = t.nzsum.get();
            ge_t[k] = std::max(1, (int)std::min<uint64_t>((uint64_t)edge_grid(hub_bytes),
                                                        (t.nchunks + 32 * run - 1) / (32 * run)));
            fg_t[k] = (int)grid1d(std::max<uint32_t>(t.nsplit, 1), 32) + (int)((t.nlong + FIX_WARPS - 1) / FIX_WARPS);
        }
    }

    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));
    const bool time_sweeps = (p->flags & GCG_PR_TIME_SWEEPS) != 0;
    std::vector<cudaEvent_t> sweep_ev; /* pairs around each edge kernel */

    /* Sweeps are queued in chunks; after each chunk the done flag is copied to
     * pinned memory. The host waits on the chunk before last, so the GPU always
     * has work queued; sweeps queued past convergence return immediately. */
    const int CHUNK = 4;
    int *h_flags = w.h_flags;
    std::vector<cudaEvent_t> chunk_ev;
    int launched = 0, stop = 0;
    int status = GCG_OK;
    while (launched < max_sweeps && !stop) {
        int n = std::min(CHUNK, max_sweeps - launched);
        for (int k = 0; k < n; ++k) {
            const int sw = launched + k;
            a.c_old = c.get() + (size_t)(sw & 1) * cstride;
            a.tex_old = w.tex[sw & 1];
            a.c_new = c.get() + (size_t)((sw + 1) & 1) * cstride;
            a.r_nz_old = rnz.get() + (size_t)(sw & 1) * pl.nnz;
            a.r_nz_new = rnz.get() + (size_t)((sw + 1) & 1) * pl.nnz;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (time_sweeps) {
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, s);
            }
            if (ntiers > 1) { /* every tier's edge pass, then every tier's fix-up */
                for (int k = 0; k < ntiers; ++k) {
                    at[k].c_old = a.c_old + g->cplan->tiers.t[k].first;
                    at[k].tex_old = k == 0 ? a.tex_old : 0ull;
                    at[k].done = a.done;
                    launch_edges(ge_t[k], hub_bytes, s, at[k]);
                }
            } else {
                launch_edges(ge, hub_bytes, s, a);
            }
            if (time_sweeps) {
                cudaEventRecord(e1, s);
                sweep_ev.push_back(e0);
                sweep_ev.push_back(e1);
            }
            if (ntiers > 1) {
                for (int k = 0; k < ntiers; ++k) launch_pdl(k_pr_fix, fg_t[k], 256, 0, s, at[k]);
            } else {
                launch_pdl(k_pr_fix, fg, 256, 0, s, a);
            }
            launch_pdl(k_pr_vertex, gv, 256, 0, s, a, sw, sw < 2 ? 1 : 0);
        }
        launched += n;
        if (cudaGetLastError() != cudaSuccess) {
            status = fail(GCG_ERR_CUDA, "pagerank sweep launch failed");
            break;
        }
        if (p->tol > 0.0) {
            int slot = (int)chunk_ev.size() % 64;
            cudaMemcpyAsync(h_flags + slot, a.done, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaEvent_t e;
            cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            cudaEventRecord(e, s);
            chunk_ev.push_back(e);
            /* wait for the previous chunk's flag */
            if (chunk_ev.size() >= 2) {
                size_t idx = chunk_ev.size() - 2;
                cudaEventSynchronize(chunk_ev[idx]);
                if (h_flags[idx % 64]) stop = 1;
            }
        }
    }
    GCG_CUDA(cudaEventRecord(ev1, s));
    GCG_CUDA(cudaEventSynchronize(ev1));
    for (auto e : chunk_ev) cudaEventDestroy(e);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (status != GCG_OK) {
        for (auto e : sweep_ev) cudaEventDestroy(e);
        return status;
    }

    uint32_t h_ctl[4]; /* ticket, done, sweeps_done, err */
    GCG_CUDA(cudaMemcpy(h_ctl, ctl.get(), sizeof(h_ctl), cudaMemcpyDeviceToHost));
    if (h_ctl[3]) {
        for (auto e : sweep_ev) cudaEventDestroy(e);
        return fail(GCG_ERR_TIMEOUT, "pagerank: the shared-memory hub copy did not complete");
    }
    const int sweeps = (int)h_ctl[2];
    const int done = (int)h_ctl[1];
    double sweep_ms = 0.0;
    int timed = 0;
    for (size_t i = 0; i + 1 < sweep_ev.size(); i += 2) {
        if ((int)(i / 2) < sweeps) { /* launches after convergence returned at once: not counted */
            float t = 0.0f;
            cudaEventElapsedTime(&t, sweep_ev[i], sweep_ev[i + 1]);
            sweep_ms += t;
            ++timed;
        }
        cudaEventDestroy(sweep_ev[i]);
        cudaEventDestroy(sweep_ev[i + 1]);
    }
    double last_res = 0.0;
    GCG_CUDA(cudaMemcpy(&last_res, a.last_res, sizeof(double), cudaMemcpyDeviceToHost));
    if (p->residuals && sweeps > 0) GCG_TRY(copy_out(p->residuals, dres.get(), (size_t)sweeps * sizeof(double), s));
    if (p->delta_log && sweeps > 0)
        GCG_TRY(copy_out(p->delta_log, dres.get() + max_sweeps + 1, (size_t)sweeps * sizeof(double), s));
    if (p->work_log && sweeps > 0) { /* every vertex updated and every in-edge gathered per sweep */
        std::vector<uint64_t> wl(2 * (size_t)sweeps);
        for (int i = 0; i < sweeps; ++i) {
            wl[2 * i] = (uint64_t)nv * (uint64_t)(i + 1);
            wl[2 * i + 1] = g->ne * (uint64_t)(i + 1);
        }
        GCG_TRY(copy_out(p->work_log, wl.data(), wl.size() * sizeof(uint64_t), s));
        GCG_CUDA(cudaStreamSynchronize(s));
    }
    if (sweeps > 0) {
        const float t = (float)p->teleport; /* teleport + damping * 0 */
        k_pr_scatter<<<grid1d(nv, 8), 256, 0, s>>>(pl.nnz, pl.nzero, pl.nz_rows.get(), pl.zero_rows.get(),
                                                  rnz.get() + (size_t)(sweeps & 1) * pl.nnz, t, p->source,
                                                  r.get());
        GCG_LAUNCH_CHECK();
    }
    if (out_rank) GCG_TRY(copy_out(out_rank, r.get(), (size_t)nv * sizeof(float), s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->sweeps = sweeps;
        stats->converged = done;
        stats->residual = last_res;
        stats->device_ms = ms;
        stats->sweep_kernel_ms = sweep_ms;
        stats->timed_sweeps = timed;
        stats->kernel_launches = 1 + (2 * ntiers + 1) * launched;
    }
    return GCG_OK;
}

}  // namespace gcg

using namespace gcg;

extern "C" {

void gcg_pr_params_default(gcg_pr_params *p) {
    if (!p) return;
    p->mode = GCG_PR_JACOBI;
    p->max_sweeps = 3;
    p->teleport = 0.15;
    p->damping = 0.85;
    p->tol = 0.0;
    p->init = 1.0f;
    p->flags = 0u;
    p->init_rank = nullptr;
    p->residuals = nullptr;
    p->source = GCG_NO_SOURCE;
    p->reserved2 = 0u;
    p->delta_log = nullptr;
    p->work_log = nullptr;
    p->delta_threshold = 0.0;
}

int gcg_pagerank_set_config(gcg_graph *g, uint32_t hub_entries, uint32_t chunk_run) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_pagerank_set_config: null graph");
    if (chunk_run == 0 || chunk_run > (1u << 16)) return fail(GCG_ERR_INVALID, "gcg_pagerank_set_config: chunk_run must be 1..65536");
    GCG_TRY(ensure_chunk_plan(g));
    g->cplan->tune_hub = hub_entries;
    g->cplan->tune_run = chunk_run;
    return GCG_OK;
}

int gcg_pagerank_set_tiers(gcg_graph *g, uint32_t tiers) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_pagerank_set_tiers: null graph");
    if (tiers < 1 || tiers > (uint32_t)MAX_TIERS) return fail(GCG_ERR_INVALID, "gcg_pagerank_set_tiers: tiers must be 1..4");
    GCG_TRY(ensure_chunk_plan(g));
    g->cplan->tune_tiers = tiers;
    return GCG_OK;
}

int gcg_pagerank_get_tiers(gcg_graph *g, uint32_t *tiers) {
    if (!g || !tiers) return fail(GCG_ERR_INVALID, "gcg_pagerank_get_tiers: null argument");
    GCG_TRY(ensure_chunk_plan(g));
    *tiers = g->cplan->tune_tiers;
    return GCG_OK;
}

int gcg_pagerank_get_config(gcg_graph *g, uint32_t *hub_entries, uint32_t *chunk_run) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_pagerank_get_config: null graph");
    GCG_TRY(ensure_chunk_plan(g));
    if (hub_entries) *hub_entries = std::min(g->cplan->hub, g->cplan->tune_hub);
    if (chunk_run) *chunk_run = g->cplan->tune_run;
    return GCG_OK;
}

int gcg_pagerank_autotune(gcg_graph *g, int sweeps, uint32_t *hub_entries, uint32_t *chunk_run, double *ms_per_sweep) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_pagerank_autotune: null graph");
    if (sweeps < 1) return fail(GCG_ERR_INVALID, "gcg_pagerank_autotune: sweeps must be >= 1");
    GCG_TRY(ensure_chunk_plan(g));
    ChunkPlan &pl = *g->cplan;
    std::vector<uint32_t> hubs;
    for (uint32_t h : {0u, 16384u, 32768u, HUB_DEFAULT, HUB_MAX})
        if (h <= pl.hub && std::find(hubs.begin(), hubs.end(), h) == hubs.end()) hubs.push_back(h);
    if (std::find(hubs.begin(), hubs.end(), pl.hub) == hubs.end()) hubs.push_back(pl.hub);
    const uint32_t runs[] = {1u, 2u, 4u, 16u};
    gcg_pr_params p;
    gcg_pr_params_default(&p);
    p.max_sweeps = sweeps;
    p.tol = 0.0;
    tbuf<float> out;
    GCG_TRY(out.alloc(std::max<uint32_t>(g->nv, 1), g->stream));
    /* each candidate: the device time of `sweeps` whole sweeps (edge pass(es),
     * fix-ups, vertex pass), best of two runs (the first also warms caches) */
    auto time_config = [&](double &t) -> int {
        t = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            gcg_pr_stats st;
            GCG_TRY(pagerank_jacobi(g, &p, out.get(), &st));
            if (st.sweeps > 0) t = std::min(t, st.device_ms / st.sweeps);
        }
        return GCG_OK;
    };
    double best = 1e300;
    uint32_t bh = std::min(pl.hub, HUB_DEFAULT), br = RUN_DEFAULT, bt = 1;
    pl.tune_tiers = 1;
    for (uint32_t h : hubs)
        for (uint32_t r : runs) {
            pl.tune_hub = h;
            pl.tune_run = r;
            double t;
            GCG_TRY(time_config(t));
            if (t < best) {
                best = t;
                bh = h;
                br = r;
            }
        }
    /* then source tiers of the chosen hub width, when the graph has sources past it */
    pl.tune_hub = bh;
    pl.tune_run = br;
    const uint32_t w = std::min(pl.hub, bh) & ~3u;
    for (uint32_t tiers = 2; w > 0 && tiers <= (uint32_t)MAX_TIERS && (uint64_t)(tiers - 1) * w < g->nv; ++tiers) {
        pl.tune_tiers = tiers;
        double t;
        GCG_TRY(time_config(t));
        if (t < best) {
            best = t;
            bt = tiers;
        }
    }
    pl.tune_tiers = bt;
    if (hub_entries) *hub_entries = bh;
    if (chunk_run) *chunk_run = br;
    if (ms_per_sweep) *ms_per_sweep = best;
    return GCG_OK;
}

int gcg_pagerank(gcg_graph *g, const gcg_pr_params *params, float *out_rank, gcg_pr_stats *stats) {
    if (!g || !params) return fail(GCG_ERR_INVALID, "gcg_pagerank: null argument");
    if (stats) *stats = gcg_pr_stats{};
    if (params->max_sweeps < 0) return fail(GCG_ERR_INVALID, "gcg_pagerank: max_sweeps < 0");
    if (params->source != GCG_NO_SOURCE && params->source >= g->nv)
        return fail(GCG_ERR_INVALID, "gcg_pagerank: personalisation source >= num_vertices");
    if (params->source != GCG_NO_SOURCE && params->mode != GCG_PR_JACOBI)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_pagerank: personalisation needs GCG_PR_JACOBI");
    if (params->mode == GCG_PR_JACOBI) return pagerank_jacobi(g, params, out_rank, stats);
    if (params->mode == GCG_PR_GS_EXACT || params->mode == GCG_PR_GS_EDGE)
        return pagerank_gs_exact(g, params, out_rank, stats);
    if (params->mode == GCG_PR_DELTA) return pagerank_delta(g, params, out_rank, stats);
    return fail(GCG_ERR_INVALID, "gcg_pagerank: unknown mode");
}

}  // extern "C"
