/*
 * Triangle counting: replaces order_by_degree + the dynamic-graph engine running
 * TriangleCountingProgram + sum_vertices / 3
 * (src/preprocessing/util/orderbydegree.hpp:59-143,
 *  example_apps/trianglecounting.cpp:95-357, :476-477).
 *
 * Device form:
 *   1. rank vertices by (in+out degree, id) ascending with one radix sort
 *      (orderbydegree.hpp:16-25, 71-89): vertexmap[v] = rank.
 *   2. orient every edge from the lower to the higher rank, radix sort and
 *      deduplicate (reciprocal edges collapse, like the reference's lastvid
 *      checks, trianglecounting.cpp:182,309) -> CSR of higher-ranked neighbours,
 *      each list ascending.
 *   3. one warp per vertex a; for each b in N+(a) the shorter of N+(a) after b
 *      and N+(b) is searched element by element in the longer, the searches of
 *      32 b's dealt evenly to the lanes (two long lists are merged by the warp
 *      instead). A match c is a triangle (a,b,c): c's
 *      count is bumped per match, b's and a's by the match totals (counts of
 *      the top-ranked vertices gathered in shared memory first) — the
 *      per-rank incident-triangle counts of <base>_degord.4B.vout.
 * Algorithmic traffic (whole count): 4*sum_{(a,b)}(d+(a)+d+(b)) + 4*E+ + 4*V.
 */
#include <algorithm>

#include "gcg_internal.cuh"
#include "gcg_mergepath.cuh"

namespace gcg {
namespace {

inline unsigned vgrid(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * 16;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

__global__ void k_degree_keys(const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ outdeg, uint32_t nv,
                              uint32_t vbits, uint64_t *__restrict__ keys, uint32_t *maxdeg) {
    uint32_t m = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint64_t d = (uint64_t)indeg[v] + outdeg[v];
        keys[v] = (d << vbits) | v;
        m = max(m, d > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxdeg, m);
}

__global__ void k_rank_scatter(const uint64_t *__restrict__ sorted, uint32_t nv, uint32_t vbits,
                               uint32_t *__restrict__ rank) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        rank[(uint32_t)(sorted[i] & mask)] = i;
}

/* key of edge e (row v, source u): (min rank << vbits) | max rank */
__global__ void __launch_bounds__(MP_THREADS) k_orient_keys(const uint32_t *__restrict__ rowptr,
                                                            const uint32_t *__restrict__ col,
                                                            const uint32_t *__restrict__ tile_row,
                                                            const uint32_t *__restrict__ tile_edge, uint32_t ntiles,
                                                            const uint32_t *__restrict__ rank, uint32_t vbits, int half,
                                                            uint32_t *__restrict__ count, uint64_t *__restrict__ keys) {
    __shared__ uint32_t s_rowend[MP_TILE];
    __shared__ uint32_t s_wsum[MP_THREADS / 32];
    __shared__ uint32_t s_base;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t r0 = tile_row[t], r1 = tile_row[t + 1];
        const uint32_t e0 = tile_edge[t], e1 = tile_edge[t + 1];
        const uint32_t nrows = r1 - r0, nedges = e1 - e0;
        for (uint32_t k = threadIdx.x; k < nrows; k += MP_THREADS) s_rowend[k] = rowptr[r0 + k + 1] - e0;
        __syncthreads();
        const uint32_t items = nrows + nedges;
        const uint32_t d0 = min((uint32_t)threadIdx.x * MP_ITEMS, items);
        const uint32_t d1 = min(d0 + MP_ITEMS, items);
        const uint32_t ti0 = mp_search(s_rowend, nrows, nedges, d0);
        if (!half) {
            uint32_t ti = ti0, tj = d0 - ti0;
            for (uint32_t d = d0; d < d1; ++d) {
                if (ti < nrows && s_rowend[ti] <= tj) {
                    ++ti;
                } else {
                    uint64_t a = rank[__ldg(col + e0 + tj)], b = rank[r0 + ti];
                    keys[e0 + tj] = a < b ? ((a << vbits) | b) : ((b << vbits) | a);
                    ++tj;
                }
            }
        } else {
            /* symmetric graph: every edge is stored both ways and both give the
             * same key, so only the copy in the higher-ranked endpoint's row is
             * kept, compacted: count, block prefix sum, one global claim per
             * tile, write (the sort that follows fixes the order) */
            uint32_t kept = 0;
            {
                uint32_t ti = ti0, tj = d0 - ti0;
                for (uint32_t d = d0; d < d1; ++d) {
                    if (ti < nrows && s_rowend[ti] <= tj) {
                        ++ti;
                    } else {
                        kept += rank[__ldg(col + e0 + tj)] <= rank[r0 + ti];
                        ++tj;
                    }
                }
            }
            uint32_t incl = kept;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            if (lane == 31) s_wsum[w] = incl;
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t run = 0;
                for (uint32_t k = 0; k < MP_THREADS / 32; ++k) {
                    const uint32_t x = s_wsum[k];
                    s_wsum[k] = run;
                    run += x;
                }
                s_base = run ? atomicAdd(count, run) : 0u;
            }
            __syncthreads();
            uint64_t pos = (uint64_t)s_base + s_wsum[w] + (incl - kept);
            uint32_t ti = ti0, tj = d0 - ti0;
            for (uint32_t d = d0; d < d1; ++d) {
                if (ti < nrows && s_rowend[ti] <= tj) {
                    ++ti;
                } else {
                    const uint64_t a = rank[__ldg(col + e0 + tj)], b = rank[r0 + ti];
                    if (a <= b) keys[pos++] = (a << vbits) | b;
                    ++tj;
                }
            }
        }
        __syncthreads();
    }
}

/* One halving of the search for the last element <= x in the sorted,
 * duplicate-free cl[base .. base + n), n >= 2: the range that still holds that
 * element shrinks to ceil(n / 2) values. After ceil(log2 n) halvings n is 1 and
 * x is present exactly when cl[base] equals it. */
__device__ __forceinline__ uint32_t last_le_step(const uint32_t *__restrict__ cl, uint32_t base, uint32_t &n,
                                                 uint32_t x) {
    const uint32_t h = n >> 1;
    if (__ldg(cl + base + h) <= x) base += h;
    n -= h;
    return base;
}

constexpr uint32_t TC_WARPS = 32;   /* 1024-thread blocks, two per SM */
constexpr uint32_t TC_TOP = 16384;  /* per-block shared counters for the top-ranked vertices */
constexpr uint32_t TC_SPLIT = 64;   /* top-range vertices with more higher-ranked neighbours go batch by batch */

/* Longest higher-ranked neighbour list among rows lo .. nv - 1 (atomicMax into *out). */
__global__ void k_max_rowlen(const uint32_t *__restrict__ rp, uint32_t lo, uint32_t nv, uint32_t *out) {
    uint32_t m = 0;
    for (uint32_t r = lo + blockIdx.x * blockDim.x + threadIdx.x; r < nv; r += gridDim.x * blockDim.x)
        m = max(m, rp[r + 1] - rp[r]);
    m = __reduce_max_sync(0xFFFFFFFFu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

/* Triangles through vertex a, 32 of its higher-ranked neighbours b at a time (a
 * batch). For each b the shorter of (N+(a) after b) and N+(b) is searched element
 * by element in the longer; the searches of the batch's b's are laid end to end
 * (a warp prefix sum of their lengths) and dealt to the lanes two at a time, so
 * every lane runs two independent searches whatever the lengths. A match c is the
 * triangle (a, b, c): c's count is bumped per match, b's by its match total, a's
 * by the batch's sum. A b whose two lists are both long is not searched: the
 * whole warp merges the two lists instead, after the searches.
 * Work is spread two ways. Vertex a goes to warp (a mod warps), numbered block
 * fastest, so the heavy vertices, which sit together in the upper ranks, land on
 * every SM. Vertices among the top `nsplit` ranks with more than TC_SPLIT
 * higher-ranked neighbours are not taken whole: their batches are dealt out one
 * by one after the other vertices, so no warp is left with a whole heavy vertex.
 * Ranks grow with degree, so the highest-ranked vertex of a triangle is nearly
 * always among the top few thousand ranks: their counts are kept in the block's
 * shared memory (dynamic, `top` entries for ranks nv - top .. nv - 1) and added
 * to `cnt` once at the end, which keeps the per-triangle increments off a few
 * hot global addresses. */
__global__ void __launch_bounds__(1024, 2) k_tc_count(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ cl,
                                                      uint32_t nv, uint32_t top, uint32_t nsplit,
                                                      const uint32_t *__restrict__ split_maxlen,
                                                      uint32_t *__restrict__ cnt, unsigned long long *total) {
    extern __shared__ uint32_t s_top[];
    __shared__ uint32_t s_pre[TC_WARPS][32], s_so[TC_WARPS][32], s_lo[TC_WARPS][32], s_nl[TC_WARPS][32],
        s_hit[TC_WARPS][32];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t *pre = s_pre[w], *so_ = s_so[w], *lo_ = s_lo[w], *nl_ = s_nl[w], *hit = s_hit[w];
    const uint32_t warp = w * gridDim.x + blockIdx.x;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lo_top = nv - top, lo_split = nv - nsplit;
    for (uint32_t i = threadIdx.x; i < top; i += blockDim.x) s_top[i] = 0;
    __syncthreads();
    auto bump = [&](uint32_t v, uint32_t inc) {
        if (v >= lo_top)
            atomicAdd(s_top + (v - lo_top), inc);
        else
            atomicAdd(cnt + v, inc);
    };
    /* the batch of a's neighbours j0 .. j0 + 31 (ab <= j0, j0 + 1 < ae); returns
     * this lane's b's match total (0 for lanes past the list) */
    auto batch = [&](uint32_t ab, uint32_t ae, uint32_t j0) -> uint32_t {
        const uint32_t j = j0 + lane;
        uint32_t ns = 0, so = 0, lo = 0, nl = 0, b = 0;
        bool mrg = false;
        if (j + 1 < ae) {
            b = __ldg(cl + j);
            const uint32_t na = ae - j - 1, bb = __ldg(rp + b), nb = __ldg(rp + b + 1) - bb;
            if (nb) {
                if (na <= nb) {
                    ns = na, so = j + 1, lo = bb, nl = nb;
                } else {
                    ns = nb, so = bb, lo = j + 1, nl = na;
                }
                /* both lists long: a merge of the two (a warp walking na + nb
                 * values, one partition search per lane) when the ns searches of
                 * log2(nl) steps would take more than three steps per merged value
                 * (a merge step is a dependent load; 1.5, 2, 3, 4 and 6 were
                 * measured) */
                const uint32_t tot = na + nb;
                if (ns * (32 - __clz((nl - 1) | 1)) > 3 * tot + 32 * (32 - __clz((tot - 1) | 1))) {
                    mrg = true, ns = 0;
                }
            }
        }
        uint32_t inc = ns;
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, inc, o);
            if (lane >= o) inc += t;
        }
        const uint32_t W = __shfl_sync(FULL, inc, 31);
        const uint32_t merges = __ballot_sync(FULL, mrg);
        if (W == 0 && merges == 0) return 0u;
        pre[lane] = inc, so_[lane] = so, lo_[lane] = lo, nl_[lane] = nl, hit[lane] = 0;
        __syncwarp();
        for (uint32_t t0 = 0; t0 < W; t0 += 64) {
            uint32_t x[2], base[2], n[2], q[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const uint32_t t = t0 + 32 * u + lane;
                n[u] = 0, x[u] = 0, base[u] = 0, q[u] = 0;
                if (t < W) {
                    /* owner: how many of the 32 inclusive prefix sums are <= t
                     * (t < W = pre[31], so at most 31; indexes stay below 31) */
                    uint32_t qq = 0;
#pragma unroll
                    for (uint32_t st = 16; st; st >>= 1)
                        if (pre[qq + st - 1] <= t) qq += st;
                    const uint32_t k = t - (qq ? pre[qq - 1] : 0);
                    x[u] = __ldg(cl + so_[qq] + k);
                    base[u] = lo_[qq], n[u] = nl_[qq], q[u] = qq;
                }
            }
            while (n[0] > 1 || n[1] > 1) {
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (n[u] > 1) base[u] = last_le_step(cl, base[u], n[u], x[u]);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u)
                if (n[u] == 1 && __ldg(cl + base[u]) == x[u]) {
                    bump(x[u], 1u);
                    atomicAdd(hit + q[u], 1u);
                }
        }
        __syncwarp();
        /* the merged pairs, one at a time by the whole warp: A = N+(a) after b,
         * B = N+(b); lane l walks diagonals [l per, (l + 1) per) of the merge that
         * takes A[i] when A[i] <= B[j], so B[j] is the least B value not below
         * A[i] and A[i] is in B exactly when they are equal */
        for (uint32_t m = merges; m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            const uint32_t jl = j0 + (uint32_t)l, A = jl + 1, na = ae - jl - 1;
            const uint32_t bl = __shfl_sync(FULL, b, l), B = __ldg(rp + bl), nb = __ldg(rp + bl + 1) - B;
            const uint32_t tot = na + nb, per = (tot + 31) / 32;
            const uint32_t d0 = min(lane * per, tot), d1 = min(d0 + per, tot);
            uint32_t i = d0 > nb ? d0 - nb : 0, hi = min(d0, na);
            while (i < hi) { /* first i with A[i] > B[d0 - 1 - i] */
                const uint32_t mid = (i + hi) >> 1;
                if (__ldg(cl + A + mid) <= __ldg(cl + B + d0 - 1 - mid))
                    i = mid + 1;
                else
                    hi = mid;
            }
            uint32_t k = d0 - i, found = 0;
            uint32_t av = i < na ? __ldg(cl + A + i) : 0u, bv = k < nb ? __ldg(cl + B + k) : 0u;
            for (uint32_t d = d0; d < d1; ++d) {
                if (i < na && (k >= nb || av <= bv)) {
                    if (k < nb && av == bv) {
                        bump(av, 1u);
                        ++found;
                    }
                    ++i;
                    if (i < na) av = __ldg(cl + A + i);
                } else {
                    ++k;
                    if (k < nb) bv = __ldg(cl + B + k);
                }
            }
            found = __reduce_add_sync(FULL, found);
            if (lane == 0 && found) hit[l] += found;
            __syncwarp();
        }
        const uint32_t h = hit[lane];
        if (h) bump(b, h);
        __syncwarp(); /* the tables are rewritten by the next batch */
        return h;
    };
    unsigned long long mine = 0;
    auto finish = [&](uint32_t a, uint32_t acc) {
        const uint32_t A = __reduce_add_sync(FULL, acc);
        if (A && lane == 0) {
            bump(a, A);
            mine += A;
        }
    };
    for (uint32_t a = warp; a < nv; a += nwarps) {
        const uint32_t ab = __ldg(rp + a), ae = __ldg(rp + a + 1);
        if (ae - ab < 2) continue; /* a triangle needs two higher-ranked neighbours */
        if (a >= lo_split && ae - ab > TC_SPLIT) continue; /* dealt out batch by batch below */
        uint32_t acc = 0;
        for (uint32_t j0 = ab; j0 + 1 < ae; j0 += 32) acc += batch(ab, ae, j0);
        finish(a, acc);
    }
    /* the split vertices' batches: item t is batch t / nsplit of vertex
     * lo_split + t % nsplit, and goes to warp t mod warps (neighbouring vertices'
     * batches to different warps); each lane checks one of its warp's items, the
     * warp runs the real ones */
    const uint64_t items = (uint64_t)nsplit * ((*split_maxlen + 31) / 32);
    for (uint64_t k0 = 0; warp + (uint64_t)nwarps * k0 < items; k0 += 32) {
        const uint64_t t = warp + (uint64_t)nwarps * (k0 + lane);
        uint32_t a = 0, ab = 0, ae = 0, j0 = 0;
        bool real = false;
        if (t < items) {
            a = lo_split + (uint32_t)(t % nsplit);
            ab = __ldg(rp + a), ae = __ldg(rp + a + 1);
            j0 = ab + 32u * (uint32_t)(t / nsplit);
            real = ae - ab > TC_SPLIT && j0 + 1 < ae;
        }
        for (uint32_t m = __ballot_sync(FULL, real); m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            const uint32_t va = __shfl_sync(FULL, a, l), vab = __shfl_sync(FULL, ab, l),
                           vae = __shfl_sync(FULL, ae, l), vj0 = __shfl_sync(FULL, j0, l);
            finish(va, batch(vab, vae, vj0));
        }
    }
    if (lane == 0 && mine) atomicAdd(total, mine);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < top; i += blockDim.x)
        if (s_top[i]) atomicAdd(cnt + lo_top + i, s_top[i]);
}

}  // namespace
}  // namespace gcg

using namespace gcg;

extern "C" int gcg_triangle_count(gcg_graph *g, uint64_t *total, uint32_t *per_rank, uint32_t *vertexmap,
                                  gcg_tc_stats *stats) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_triangle_count: null graph");
    GCG_TRY(ensure_plan(g));
    cudaStream_t s = g->stream;
    const uint32_t nv = g->nv, vbits = g->vbits;
    const uint64_t ne = g->ne;
    const PrPlan &pl = *g->plan;

    cudaEvent_t ev0, ev1;
    GCG_CUDA(cudaEventCreate(&ev0));
    GCG_CUDA(cudaEventCreate(&ev1));
    GCG_CUDA(cudaEventRecord(ev0, s));

    /* 1. degree ranking */
    tbuf<uint64_t> keys, tmp;
    tbuf<uint32_t> rank, dmax;
    GCG_TRY(keys.alloc(std::max<uint64_t>(nv, ne), s));
    GCG_TRY(tmp.alloc(std::max<uint64_t>(nv, ne), s));
    GCG_TRY(rank.alloc(nv, s));
    GCG_TRY(dmax.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(dmax.get(), 0, 4, s));
    k_degree_keys<<<vgrid(nv), 256, 0, s>>>(g->indeg.get(), g->outdeg.get(), nv, vbits, keys.get(), dmax.get());
    uint32_t maxdeg = 0;
    GCG_CUDA(cudaMemcpyAsync(&maxdeg, dmax.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    uint32_t dbits = 1;
    while (dbits < 33 && (1ull << dbits) <= maxdeg) ++dbits;
    if (vbits + dbits > 64) return fail(GCG_ERR_UNSUPPORTED, "gcg_triangle_count: degree and id do not fit 64 bits");
    uint64_t *sorted = nullptr;
    GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nv, 0, (int)(vbits + dbits), &sorted, s));
    k_rank_scatter<<<vgrid(nv), 256, 0, s>>>(sorted, nv, vbits, rank.get());
    GCG_LAUNCH_CHECK();

    /* 2. oriented, deduplicated edges in rank space */
    uint64_t m_or = 0;
    dbuf<uint32_t> rp, cl;
    GCG_TRY(rp.alloc((size_t)nv + 1));
    if (ne > 0) {
        int per_sm = 4;
        unsigned tb = (unsigned)std::max<uint32_t>(1, std::min<uint32_t>(pl.ntiles, (uint32_t)(num_sms() * per_sm)));
        /* a symmetric graph keeps one of the two stored copies of every edge */
        const int half = g->symmetric ? 1 : 0;
        tbuf<uint32_t> fl, d_tot;
        GCG_TRY(d_tot.alloc(1, s));
        GCG_CUDA(cudaMemsetAsync(d_tot.get(), 0, 4, s));
        k_orient_keys<<<tb, MP_THREADS, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), pl.tile_row.get(),
                                               pl.tile_edge.get(), pl.ntiles, rank.get(), vbits, half, d_tot.get(),
                                               keys.get());
        GCG_LAUNCH_CHECK();
        uint64_t nk = ne;
        if (half) {
            uint32_t kept = 0;
            GCG_CUDA(cudaMemcpyAsync(&kept, d_tot.get(), 4, cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            nk = kept;
        }
        if (nk > 0) {
            GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nk, 0, 2 * (int)vbits, &sorted, s));
            /* unique: flags + scan + scatter, then CSR by the low-rank half */
            GCG_TRY(fl.alloc(nk, s));
            uint64_t *other = sorted == keys.get() ? tmp.get() : keys.get();
            GCG_TRY(unique_u64(sorted, nk, fl.get(), d_tot.get(), other, s));
            uint32_t tot = 0;
            GCG_CUDA(cudaMemcpyAsync(&tot, d_tot.get(), 4, cudaMemcpyDeviceToHost, s));
            GCG_CUDA(cudaStreamSynchronize(s));
            m_or = tot;
            GCG_TRY(cl.alloc(m_or));
            GCG_TRY(csr_from_sorted_keys(other, m_or, vbits, nv, rp.get(), cl.get(), s));
        } else {
            GCG_TRY(cl.alloc(1));
            GCG_CUDA(cudaMemsetAsync(rp.get(), 0, ((size_t)nv + 1) * 4, s));
        }
    } else {
        GCG_TRY(cl.alloc(1));
        GCG_CUDA(cudaMemsetAsync(rp.get(), 0, ((size_t)nv + 1) * 4, s));
    }

    /* 3. count */
    tbuf<uint32_t> cnt;
    tbuf<unsigned long long> d_total;
    uint32_t *cnt_ptr;
    const bool dev_counts = per_rank && is_device_ptr(per_rank);
    if (dev_counts) {
        cnt_ptr = per_rank;
    } else {
        GCG_TRY(cnt.alloc(nv, s));
        cnt_ptr = cnt.get();
    }
    GCG_TRY(d_total.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(cnt_ptr, 0, (size_t)nv * 4, s));
    GCG_CUDA(cudaMemsetAsync(d_total.get(), 0, 8, s));
    /* persistent: two 1024-thread blocks per SM, each with its own top-rank counters */
    const uint32_t top = std::min(nv, TC_TOP);
    const uint32_t nsplit = std::min(nv, std::max<uint32_t>(65536u, nv / 16));
    tbuf<uint32_t> split_maxlen;
    GCG_TRY(split_maxlen.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(split_maxlen.get(), 0, 4, s));
    if (nsplit) {
        k_max_rowlen<<<vgrid(nsplit), 256, 0, s>>>(rp.get(), nv - nsplit, nv, split_maxlen.get());
        GCG_LAUNCH_CHECK();
    }
    GCG_CUDA(cudaFuncSetAttribute(k_tc_count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(TC_TOP * 4)));
    unsigned cb = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)nv + TC_WARPS - 1) / TC_WARPS, (uint64_t)num_sms() * 2));
    k_tc_count<<<cb, TC_WARPS * 32, (size_t)top * 4, s>>>(rp.get(), cl.get(), nv, top, nsplit, split_maxlen.get(),
                                                          cnt_ptr, d_total.get());
    GCG_LAUNCH_CHECK();
    GCG_CUDA(cudaEventRecord(ev1, s));
    unsigned long long tri = 0;
    GCG_CUDA(cudaMemcpyAsync(&tri, d_total.get(), 8, cudaMemcpyDeviceToHost, s));
    if (per_rank && !dev_counts) GCG_TRY(copy_out(per_rank, cnt_ptr, (size_t)nv * 4, s));
    if (vertexmap) GCG_TRY(copy_out(vertexmap, rank.get(), (size_t)nv * 4, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (total) *total = tri;
    if (stats) {
        stats->triangles = tri;
        stats->oriented_edges = m_or;
        stats->device_ms = ms;
    }
    return GCG_OK;
}
