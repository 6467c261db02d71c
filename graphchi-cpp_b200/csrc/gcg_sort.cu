/*
 * Device radix sort and scan: the B200 replacement of the sharder's shovel sort
 * (stable LSD radix sort with 8-bit digits, src/util/radixSort.hpp:50-116, used by
 * shard_flushinfo::flush sharder.hpp:192 and finish_shard sharder.hpp:640).
 *
 * Design (HBM-bound integer work, no tensor cores):
 *   per 8-bit digit pass: upsweep (per-tile digit histogram, per-warp shared-memory
 *   counters) -> exclusive scan of the digit-major count table -> downsweep (each
 *   warp ranks its own contiguous 512 keys with warp-private digit counters and
 *   per-bit ballots, one digit-major scan over (digit, warp) gives every key its
 *   place in the tile, keys are regrouped by digit in shared memory and written so
 *   that each digit run of a tile is a contiguous, coalesced store).
 * Tiles are 4096 keys (256 threads x 16); each warp reads its 512 keys as 16
 * coalesced rounds of 32.
 */
#include <algorithm>

#include "gcg_internal.cuh"

namespace gcg {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

/* Warp w of a tile owns the contiguous keys [w*WSEG, (w+1)*WSEG) of the tile and
 * reads them as RS_ITEMS coalesced rounds of 32; keeping each warp's keys
 * contiguous lets the downsweep rank them with warp-private counters and stay
 * stable (tile order = warp order, then round, then lane). */
constexpr int RS_WSEG = RS_TILE / RS_WARPS;

__global__ void __launch_bounds__(RS_THREADS) rs_upsweep(const uint64_t *__restrict__ keys, uint64_t n,
                                                         int shift, uint32_t dmask, uint32_t ntiles,
                                                         uint32_t *__restrict__ counts) {
    __shared__ uint32_t hist[RS_WARPS][256];
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&hist[0][0])[i] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t wbase = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)warp * RS_WSEG;
    uint32_t dig[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint64_t i = wbase + (uint64_t)k * 32 + lane;
        dig[k] = (i < n) ? (uint32_t)((__ldg(keys + i) >> shift) & dmask) : 256u;
    }
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k)
        if (dig[k] < 256u) atomicAdd(&hist[warp][dig[k]], 1u);
    __syncthreads();
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s += hist[w][threadIdx.x];
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = s;
}

/* Block-wide exclusive scan of one uint32 per thread (RS_THREADS threads). */
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t *s_warp) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) s_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < RS_WARPS) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < RS_WARPS) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t before = warp ? s_warp[warp - 1] : 0u;
    return before + v - x;
}

__global__ void __launch_bounds__(RS_THREADS) rs_downsweep(const uint64_t *__restrict__ keys_in,
                                                           uint64_t *__restrict__ keys_out, uint64_t n,
                                                           int shift, uint32_t dmask, uint32_t ntiles,
                                                           const uint32_t *__restrict__ counts,
                                                           const uint32_t *__restrict__ offsets) {
    __shared__ uint64_t s_keys[RS_TILE];
    __shared__ uint32_t s_gofs[256];
    __shared__ uint32_t s_lstart[256];
    __shared__ uint32_t s_wcnt[RS_WARPS][256]; /* per warp: keys of each digit (then the warp's offset) */
    __shared__ uint32_t s_scan[RS_WARPS];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    const uint32_t tile_n = (n - base) < (uint64_t)RS_TILE ? (uint32_t)(n - base) : (uint32_t)RS_TILE;
    const uint64_t wbase = base + (uint64_t)warp * RS_WSEG;

    uint64_t key[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint64_t i = wbase + (uint64_t)k * 32 + lane;
        key[k] = (i < n) ? __ldg(keys_in + i) : 0ull;
    }
    for (int w = 0; w < RS_WARPS; ++w) s_wcnt[w][tid] = 0;
    const uint32_t gofs = offsets[(uint64_t)tid * ntiles + blockIdx.x];
    const uint32_t h = counts[(uint64_t)tid * ntiles + blockIdx.x];
    const uint32_t lstart = block_excl_scan(h, s_scan); /* synchronises: s_wcnt is clear */
    s_lstart[tid] = lstart;
    /* tile position i of digit d goes to gofs[d] + (i - lstart[d]); one table
     * instead of two (uint32 wrap-around is exact: every index is below 2^32) */
    s_gofs[tid] = gofs - lstart;

    /* warp-private ranking over the warp's 16 rounds, in key order */
    uint16_t lrank[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint64_t i = wbase + (uint64_t)k * 32 + lane;
        const bool valid = i < n;
        const uint32_t d = valid ? (uint32_t)((key[k] >> shift) & dmask) : 256u;
        /* lanes holding the same digit, from one vote per digit bit (cheaper here
         * than __match_any_sync, which competes with the shared-memory traffic) */
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t vb = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? vb : ~vb;
        }
        const uint32_t before = valid ? s_wcnt[warp][d] : 0u;
        lrank[k] = (uint16_t)(before + __popc(peers & lanemask_lt()));
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) s_wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    /* digit-major offsets: digit d's keys of warp w start after those of warps < w */
    {
        uint32_t run = s_lstart[tid];
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t c = s_wcnt[w][tid];
            s_wcnt[w][tid] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint64_t i = wbase + (uint64_t)k * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)((key[k] >> shift) & dmask);
            s_keys[s_wcnt[warp][d] + lrank[k]] = key[k];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
        const uint64_t kk = s_keys[i];
        const uint32_t d = (uint32_t)((kk >> shift) & dmask);
        keys_out[(uint32_t)(s_gofs[d] + i)] = kk;
    }
}

/* ---- scan -------------------------------------------------------------- */

constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 16;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__global__ void __launch_bounds__(SC_THREADS) sc_reduce(const uint32_t *__restrict__ in, uint64_t n,
                                                        uint32_t *__restrict__ sums) {
    __shared__ uint32_t s_warp[SC_THREADS / 32];
    const uint64_t base = (uint64_t)blockIdx.x * SC_TILE;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) {
        uint64_t i = base + (uint64_t)k * SC_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < SC_THREADS / 32; ++w) t += s_warp[w];
        sums[blockIdx.x] = t;
    }
}

/* Exclusive scan of one tile with a carried-in offset (offsets[blockIdx] or 0). */
__global__ void __launch_bounds__(SC_THREADS) sc_scan_tile(const uint32_t *in, uint32_t *out, uint64_t n,
                                                           const uint32_t *__restrict__ block_off,
                                                           uint32_t *total) {
    __shared__ uint32_t s_v[SC_TILE];
    __shared__ uint32_t s_warp[SC_THREADS / 32];
    const uint64_t base = (uint64_t)blockIdx.x * SC_TILE;
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) {
        uint64_t i = base + (uint64_t)k * SC_THREADS + tid;
        s_v[k * SC_THREADS + tid] = (i < n) ? in[i] : 0u;
    }
    __syncthreads();
    uint32_t loc[SC_ITEMS];
    uint32_t t = 0;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) {
        loc[k] = t;
        t += s_v[tid * SC_ITEMS + k];
    }
    uint32_t pre = block_excl_scan(t, s_warp);
    uint32_t off = block_off ? block_off[blockIdx.x] : 0u;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) s_v[tid * SC_ITEMS + k] = off + pre + loc[k];
    if (total && tid == SC_THREADS - 1 && (uint64_t)(blockIdx.x + 1) * SC_TILE >= n) *total = off + pre + t;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) {
        uint64_t i = base + (uint64_t)k * SC_THREADS + tid;
        if (i < n) out[i] = s_v[k * SC_THREADS + tid];
    }
}

/* ---- merge of two sorted runs (merge path) ------------------------------ */

constexpr int MG_THREADS = 256;
constexpr int MG_ITEMS = 8; /* pairwise merges of the piecewise sort */
constexpr int MG_TILE = MG_THREADS * MG_ITEMS;
constexpr int MF_ITEMS = 16; /* the fused last merge: larger tiles hide its per-tile latency */
constexpr int MF_TILE = MG_THREADS * MF_ITEMS;

/* Tiles are staged in shared memory with one pad slot after every ITEMS keys, so
 * the ITEMS consecutive keys a thread writes after merging fall on distinct banks. */
template <int ITEMS>
__device__ __forceinline__ uint32_t padx(uint32_t e) { return e + e / ITEMS; }

template <int ITEMS>
struct SView { /* keys [off, off + n) of a padded tile */
    const uint64_t *s;
    uint32_t off;
    __device__ __forceinline__ uint64_t operator[](uint32_t i) const { return s[padx<ITEMS>(off + i)]; }
};

/* how many of the first diag outputs come from a (a first on equal keys) */
template <typename A, typename B, typename I>
__device__ __forceinline__ I merge_path(const A &a, I na, const B &b, I nb, I diag) {
    I lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
    while (lo < hi) {
        const I mid = (lo + hi) >> 1;
        if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* split[t] = a's share of the first t*TILE outputs, t = 0..ntiles */
template <int TILE>
__global__ void k_merge_split(const uint64_t *__restrict__ a, uint64_t na, const uint64_t *__restrict__ b,
                              uint64_t nb, uint64_t ntiles, uint64_t *__restrict__ split) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t <= ntiles;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t d = t * TILE < na + nb ? t * TILE : na + nb;
        split[t] = merge_path(a, na, b, nb, d);
    }
}

/* Stages a tile's pieces a[a0, a0+la) and b[b0, b0+lb) in s, merges them (each
 * thread ITEMS outputs from its own merge-path split) and leaves the merged tile
 * in s (padded); v[k] = merged output dg + k of this thread. */
template <int ITEMS>
__device__ __forceinline__ void tile_merge(const uint64_t *__restrict__ a, uint64_t a0, uint32_t la,
                                           const uint64_t *__restrict__ b, uint64_t b0, uint32_t lb, uint64_t *s,
                                           uint64_t (&v)[ITEMS], uint32_t &dg) {
    const uint32_t tot = la + lb;
    for (uint32_t i = threadIdx.x; i < la; i += MG_THREADS) s[padx<ITEMS>(i)] = a[a0 + i];
    for (uint32_t i = threadIdx.x; i < lb; i += MG_THREADS) s[padx<ITEMS>(la + i)] = b[b0 + i];
    __syncthreads();
    const SView<ITEMS> sa{s, 0}, sb{s, la};
    dg = threadIdx.x * ITEMS < tot ? threadIdx.x * ITEMS : tot;
    uint32_t i = merge_path(sa, la, sb, lb, dg), j = dg - i;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        v[k] = 0;
        if (dg + k < tot) {
            const bool take_a = i < la && (j >= lb || sa[i] <= sb[j]);
            v[k] = take_a ? sa[i] : sb[j];
            if (take_a) ++i; else ++j;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
        if (dg + k < tot) s[padx<ITEMS>(dg + k)] = v[k];
    __syncthreads();
}

/* One output tile per block, written back with coalesced stores. */
__global__ void __launch_bounds__(MG_THREADS) k_merge_u64(const uint64_t *__restrict__ a, uint64_t na,
                                                          const uint64_t *__restrict__ b, uint64_t nb,
                                                          const uint64_t *__restrict__ split,
                                                          uint64_t *__restrict__ out) {
    __shared__ uint64_t s_in[MG_TILE + MG_TILE / MG_ITEMS];
    const uint64_t n = na + nb;
    const uint64_t d0 = (uint64_t)blockIdx.x * MG_TILE;
    const uint64_t d1 = d0 + MG_TILE < n ? d0 + MG_TILE : n;
    const uint64_t a0 = split[blockIdx.x], a1 = split[blockIdx.x + 1];
    const uint64_t b0 = d0 - a0, b1 = d1 - a1;
    const uint32_t la = (uint32_t)(a1 - a0), lb = (uint32_t)(b1 - b0), tot = la + lb;
    uint64_t v[MG_ITEMS];
    uint32_t dg;
    tile_merge<MG_ITEMS>(a, a0, la, b, b0, lb, s_in, v, dg);
    for (uint32_t x = threadIdx.x; x < tot; x += MG_THREADS) out[d0 + x] = s_in[padx<MG_ITEMS>(x)];
}

/* ---- merge + unique + CSR in one pass ------------------------------------
 * The last merge of the sharder's sorted runs, the duplicate filter, the
 * compaction offsets and the CSR decode fused: each block merges one tile of
 * MF_TILE outputs (as k_merge_u64), flags the keys to keep, and finds where its
 * kept keys start in the output by a decoupled look-back over the tiles before
 * it (tiles are taken in ticket order, so a block only waits on blocks that are
 * already running; every wait is bounded and sets an error flag on expiry).
 * It then writes the column of every kept key, the row pointers of the rows
 * its keys open, optionally the kept keys themselves, and takes duplicates off
 * the raw out-degree counts. */
static_assert(MG_THREADS == RS_THREADS, "block_excl_scan is sized for RS_THREADS");
constexpr uint32_t TS_AGG = 1u, TS_INC = 2u;
constexpr long long LB_SPIN = 1ll << 22;

__device__ __forceinline__ void ts_store(unsigned long long *p, uint32_t status, uint32_t val) {
    const unsigned long long w = ((unsigned long long)status << 32) | val;
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}

__device__ __forceinline__ unsigned long long ts_load(const unsigned long long *p) {
    unsigned long long w;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}

struct FinishArgs {
    const uint64_t *a, *b;
    uint64_t na, nb, kept;
    const uint64_t *split;
    uint32_t kbits, nv;
    int dedup;
    uint32_t *rowptr, *col;
    uint64_t *keys_out;   /* kept keys, or null */
    uint32_t *outdeg_dup; /* raw out-degree counts to take duplicates off, or null */
    uint32_t *ticket;
    unsigned long long *tstate;
    uint32_t *total;
    int *err;
};

/* exclusive prefix of tile t's kept keys: warp 0 walks back over the tile states,
 * 32 at a time, until it meets an inclusive prefix */
__device__ __forceinline__ uint32_t look_back(const FinishArgs &f, uint32_t t, uint32_t lane) {
    uint32_t excl = 0;
    int64_t j = (int64_t)t - 1;
    while (j >= 0) {
        const int64_t idx = j - (int64_t)lane;
        unsigned long long w = 0;
        if (idx >= 0) {
            long long spin = 0;
            do {
                w = ts_load(f.tstate + idx);
            } while ((w >> 32) == 0 && ++spin < LB_SPIN);
            if ((w >> 32) == 0) atomicExch(f.err, 1);
        }
        const uint32_t status = (uint32_t)(w >> 32);
        const uint32_t inc = __ballot_sync(0xFFFFFFFFu, idx >= 0 && status == TS_INC);
        const uint32_t stop = inc ? (uint32_t)(__ffs(inc) - 1) : 31u; /* nearest inclusive tile */
        uint32_t v = (idx >= 0 && lane <= stop) ? (uint32_t)w : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        excl += v;
        if (inc) break;
        j -= 32;
    }
    return excl;
}

__global__ void __launch_bounds__(MG_THREADS, 4) k_merge_finish(FinishArgs f) {
    __shared__ uint64_t s_in[MF_TILE + MF_TILE / MF_ITEMS];
    __shared__ uint32_t s_warp[RS_WARPS];
    __shared__ uint32_t s_tile, s_excl, s_sum;
    if (threadIdx.x == 0) s_tile = atomicAdd(f.ticket, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint64_t n = f.na + f.nb;
    const uint64_t d0 = (uint64_t)t * MF_TILE;
    const uint64_t d1 = d0 + MF_TILE < n ? d0 + MF_TILE : n;
    const uint64_t a0 = f.split[t], a1 = f.split[t + 1];
    const uint64_t b0 = d0 - a0, b1 = d1 - a1;
    const uint32_t la = (uint32_t)(a1 - a0), lb = (uint32_t)(b1 - b0), tot = la + lb;
    uint64_t v[MF_ITEMS];
    uint32_t dg;
    tile_merge<MF_ITEMS>(f.a, a0, la, f.b, b0, lb, s_in, v, dg);
    /* the key before this thread's first: the previous thread's last, or the
     * previous tile's last (the larger of the last a and b keys before it) */
    uint64_t prev = 0;
    if (threadIdx.x == 0) {
        if (d0 > 0) {
            const uint64_t x = a0 ? f.a[a0 - 1] : 0ull, y = b0 ? f.b[b0 - 1] : 0ull;
            prev = x > y ? x : y;
        }
    } else if (dg > 0) {
        prev = s_in[padx<MF_ITEMS>(dg - 1)];
    }
    uint32_t fl = 0, cnt = 0;
    {
        uint64_t pk = prev;
#pragma unroll
        for (int k = 0; k < MF_ITEMS; ++k) {
            const uint64_t gi = d0 + dg + k;
            if (dg + k < tot && gi < f.kept) {
                const bool keep = !f.dedup || gi == 0 || v[k] != pk;
                fl |= (keep ? 1u : 0u) << k;
                cnt += keep ? 1u : 0u;
            }
            pk = v[k];
        }
    }
    const uint32_t local = block_excl_scan(cnt, s_warp);
    if (threadIdx.x == MG_THREADS - 1) {
        const uint32_t tile_sum = local + cnt;
        if (t == 0) ts_store(f.tstate, TS_INC, tile_sum);
        else ts_store(f.tstate + t, TS_AGG, tile_sum);
        s_sum = tile_sum;
    }
    __syncthreads();
    const uint32_t tile_sum = s_sum;
    if (threadIdx.x < 32) {
        uint32_t excl = 0;
        if (t > 0) {
            excl = look_back(f, t, threadIdx.x);
            if (threadIdx.x == 0) ts_store(f.tstate + t, TS_INC, excl + tile_sum);
        }
        if (threadIdx.x == 0) s_excl = excl;
    }
    __syncthreads();
    const uint64_t mask = (f.kbits >= 64) ? ~0ull : ((1ull << f.kbits) - 1ull);
    const uint32_t base = s_excl;
    /* the kept keys, compacted in shared memory (the merged tile is no longer
     * read), then written out with coalesced stores; row pointers and repeat
     * counts from the thread that holds the key */
    uint32_t q = local;
    uint64_t pk = prev;
#pragma unroll
    for (int k = 0; k < MF_ITEMS; ++k) {
        const uint64_t gi = d0 + dg + k;
        if (dg + k < tot && gi < f.kept) {
            const uint64_t key = v[k];
            const uint32_t row = (uint32_t)(key >> f.kbits);
            if ((fl >> k) & 1u) {
                s_in[padx<MF_ITEMS>(q)] = key;
                const int64_t prow = gi == 0 ? -1 : (int64_t)(pk >> f.kbits);
                for (int64_t r = prow + 1; r <= (int64_t)row; ++r) f.rowptr[r] = base + q;
                ++q;
            } else if (f.outdeg_dup) {
                atomicSub(f.outdeg_dup + (uint32_t)(key & mask), 1u);
            }
            if (gi == f.kept - 1) { /* rows after the last key end at the total */
                for (uint64_t r = (uint64_t)row + 1; r <= f.nv; ++r) f.rowptr[r] = base + q;
                *f.total = base + q;
            }
        }
        pk = v[k];
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < tile_sum; x += MG_THREADS) {
        const uint64_t key = s_in[padx<MF_ITEMS>(x)];
        f.col[base + x] = (uint32_t)(key & mask);
        if (f.keys_out) f.keys_out[base + x] = key;
    }
}

}  // namespace

int merge_u64(const uint64_t *a, uint64_t na, const uint64_t *b, uint64_t nb, uint64_t *out, cudaStream_t s) {
    const uint64_t n = na + nb;
    if (n == 0) return GCG_OK;
    if (na == 0 || nb == 0) {
        GCG_CUDA(cudaMemcpyAsync(out, na ? a : b, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        return GCG_OK;
    }
    const uint64_t ntiles = (n + MG_TILE - 1) / MG_TILE;
    if (ntiles >= 0x7FFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "merge: too many keys");
    tbuf<uint64_t> split;
    GCG_TRY(split.alloc(ntiles + 1, s));
    k_merge_split<MG_TILE><<<(unsigned)std::min<uint64_t>((ntiles + 256) / 256, (uint64_t)num_sms() * 8), 256, 0, s>>>(
        a, na, b, nb, ntiles, split.get());
    k_merge_u64<<<(unsigned)ntiles, MG_THREADS, 0, s>>>(a, na, b, nb, split.get(), out);
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

int merge_unique_csr(const uint64_t *a, uint64_t na, const uint64_t *b, uint64_t nb, uint64_t kept, bool dedup,
                     uint32_t kbits, uint32_t nv, uint32_t *rowptr, uint32_t *col, uint64_t *keys_out,
                     uint32_t *outdeg_dup, uint64_t *ne, cudaStream_t s) {
    *ne = 0;
    if (kept == 0) {
        GCG_CUDA(cudaMemsetAsync(rowptr, 0, ((size_t)nv + 1) * 4, s));
        return GCG_OK;
    }
    const uint64_t n = na + nb;
    if (kept > n || kept > 0xFFFFFFFFull) return fail(GCG_ERR_INVALID, "merge_unique_csr: bad key count");
    const uint64_t ntiles = (kept + MF_TILE - 1) / MF_TILE;
    tbuf<uint64_t> split;
    tbuf<unsigned long long> tstate;
    tbuf<uint32_t> ctl; /* ticket, total, err */
    GCG_TRY(split.alloc(ntiles + 1, s));
    GCG_TRY(tstate.alloc(ntiles, s));
    GCG_TRY(ctl.alloc(3, s));
    GCG_CUDA(cudaMemsetAsync(tstate.get(), 0, ntiles * sizeof(unsigned long long), s));
    GCG_CUDA(cudaMemsetAsync(ctl.get(), 0, 3 * sizeof(uint32_t), s));
    k_merge_split<MF_TILE><<<(unsigned)std::min<uint64_t>((ntiles + 256) / 256, (uint64_t)num_sms() * 8), 256, 0, s>>>(
        a, na, b ? b : a, nb, ntiles, split.get());
    FinishArgs f;
    f.a = a;
    f.b = b ? b : a;
    f.na = na;
    f.nb = nb;
    f.kept = kept;
    f.split = split.get();
    f.kbits = kbits;
    f.nv = nv;
    f.dedup = dedup ? 1 : 0;
    f.rowptr = rowptr;
    f.col = col;
    f.keys_out = keys_out;
    f.outdeg_dup = outdeg_dup;
    f.ticket = ctl.get();
    f.tstate = tstate.get();
    f.total = ctl.get() + 1;
    f.err = (int *)(ctl.get() + 2);
    k_merge_finish<<<(unsigned)ntiles, MG_THREADS, 0, s>>>(f);
    GCG_LAUNCH_CHECK();
    uint32_t h[2] = {0, 0};
    GCG_CUDA(cudaMemcpyAsync(h, ctl.get() + 1, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (h[1]) return fail(GCG_ERR_TIMEOUT, "merge_unique_csr: a tile's prefix never arrived");
    *ne = h[0];
    return GCG_OK;
}

int scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total_dev, cudaStream_t s) {
    if (n == 0) {
        if (total_dev) GCG_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s));
        return GCG_OK;
    }
    uint64_t nb = (n + SC_TILE - 1) / SC_TILE;
    if (nb == 1) {
        sc_scan_tile<<<1, SC_THREADS, 0, s>>>(in, out, n, nullptr, total_dev);
        GCG_LAUNCH_CHECK();
        return GCG_OK;
    }
    tbuf<uint32_t> sums;
    GCG_TRY(sums.alloc(nb, s));
    sc_reduce<<<(unsigned)nb, SC_THREADS, 0, s>>>(in, n, sums.get());
    GCG_LAUNCH_CHECK();
    GCG_TRY(scan_u32(sums.get(), sums.get(), nb, nullptr, s));
    sc_scan_tile<<<(unsigned)nb, SC_THREADS, 0, s>>>(in, out, n, sums.get(), total_dev);
    GCG_LAUNCH_CHECK();
    /* sums is released stream-ordered, after the kernels above. */
    return GCG_OK;
}

int radix_sort_u64(uint64_t *keys, uint64_t *tmp, uint64_t n, int begin_bit, int end_bit,
                   uint64_t **result, cudaStream_t s) {
    *result = keys;
    if (n <= 1 || end_bit <= begin_bit) return GCG_OK;
    if (n > 0xFFFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "radix sort: more than 2^32-1 keys");
    uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    tbuf<uint32_t> counts, offsets;
    GCG_TRY(counts.alloc((size_t)256 * ntiles, s));
    GCG_TRY(offsets.alloc((size_t)256 * ntiles, s));
    uint64_t *a = keys, *b = tmp;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        const int nb = end_bit - shift < 8 ? end_bit - shift : 8;
        const uint32_t dmask = (1u << nb) - 1u;
        rs_upsweep<<<ntiles, RS_THREADS, 0, s>>>(a, n, shift, dmask, ntiles, counts.get());
        GCG_LAUNCH_CHECK();
        GCG_TRY(scan_u32(counts.get(), offsets.get(), (uint64_t)256 * ntiles, nullptr, s));
        rs_downsweep<<<ntiles, RS_THREADS, 0, s>>>(a, b, n, shift, dmask, ntiles, counts.get(), offsets.get());
        GCG_LAUNCH_CHECK();
        uint64_t *t = a; a = b; b = t;
    }
    *result = a;
    return GCG_OK;
}

}  // namespace gcg
