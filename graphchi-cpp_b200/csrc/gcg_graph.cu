/*
 * The device sharder: edge list -> HBM-resident interval-sorted CSR blocks.
 *
 * Replaces (src/preprocessing/sharder.hpp):
 *   preprocessing_add_edge :427-446  self-loop drop, max vertex id
 *   shard_flushinfo::flush :161-202  shovel radix sort by dst       -> one device radix sort of
 *   kway_merge + add       :861-892  merge by dst, interval cuts        (dst<<b | src) keys
 *   finish_shard           :620-848  per-shard sort by src, adjacency -> stable re-sort by src
 *   degrees                :748-751, :996-1006                        -> CSR row-pointer differences
 * Intervals are cut with the sink's exact rule (a shard closes before the first
 * edge of a new destination once it holds >= edges_per_shard edges; the quota is
 * recomputed after each cut), found with binary searches over the in-CSR row
 * pointers instead of a sequential merge.
 */
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "gcg_internal.cuh"

namespace gcg {
namespace {

struct ScanInfo {
    unsigned long long kept;
    uint32_t maxid;
    uint32_t bad;
};

__global__ void k_scan_edges(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t m,
                             uint32_t nv_limit, ScanInfo *info) {
    uint32_t mx = 0, bad = 0;
    unsigned long long kept = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = src[i], d = dst[i];
        if (s == d) continue; /* sharder.hpp:428-431: self-loops never reach max_vertex_id */
        ++kept;
        mx = max(mx, max(s, d));
        if (nv_limit && (s >= nv_limit || d >= nv_limit)) bad = 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_down_sync(0xFFFFFFFFu, mx, o));
        kept += __shfl_down_sync(0xFFFFFFFFu, kept, o);
        bad |= __shfl_down_sync(0xFFFFFFFFu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (kept) atomicAdd(&info->kept, kept);
        if (mx) atomicMax(&info->maxid, mx);
        if (bad) atomicOr(&info->bad, 1u);
    }
}

/* key = (row << vbits) | col; self-loops become the all-ones sentinel, which
 * sorts after every real key (a real key never has row == col == all ones). */
__global__ void k_make_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t m,
                            uint32_t vbits, int sym, uint64_t *__restrict__ keys, uint32_t *__restrict__ outcnt) {
    const uint64_t sent = (vbits >= 32) ? ~0ull : ((1ull << (2 * vbits)) - 1ull);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = src[i], d = dst[i];
        bool self = s == d;
        keys[i] = self ? sent : ((d << vbits) | s);
        if (sym) keys[m + i] = self ? sent : ((s << vbits) | d);
        /* raw out-degrees: one count per key's source (repeats are taken off later) */
        if (outcnt && !self) {
            atomicAdd(outcnt + s, 1u);
            if (sym) atomicAdd(outcnt + d, 1u);
        }
    }
}

__global__ void k_unique_flags(const uint64_t *__restrict__ keys, uint64_t n, uint32_t *__restrict__ flags) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_unique_scatter(const uint64_t *__restrict__ keys, uint64_t n, const uint32_t *__restrict__ pos,
                                 uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (i == 0 || keys[i] != keys[i - 1]) out[pos[i]] = keys[i];
}

/* Sorted keys -> CSR: col[i] = low bits of key i; rowptr[r] = number of keys
 * whose row (high bits) is below r, found by a lower-bound search per row. Every
 * row pointer is its own thread's work, so a long run of empty rows (the
 * lowest ranks of a degree ordering are the isolated vertices) costs no more
 * than any other. */
__global__ void k_csr_from_keys(const uint64_t *__restrict__ keys, uint64_t n, uint32_t vbits, uint32_t nv,
                                uint32_t *__restrict__ rowptr, uint32_t *__restrict__ col) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    const uint64_t total = n > (uint64_t)nv + 1 ? n : (uint64_t)nv + 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i < n) col[i] = (uint32_t)(__ldg(keys + i) & mask);
        if (i <= nv) {
            uint64_t lo = 0, hi = n;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if ((__ldg(keys + mid) >> vbits) < i)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            rowptr[i] = (uint32_t)lo;
        }
    }
}

/* Swap the halves of each key: (a << b | c) -> (c << b | a). */
__global__ void k_swap_key(const uint64_t *__restrict__ in, uint64_t n, uint32_t vbits, uint64_t *__restrict__ out) {
    const uint64_t mask = (1ull << vbits) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = in[i];
        out[i] = ((k & mask) << vbits) | (k >> vbits);
    }
}

__global__ void k_degree(const uint32_t *__restrict__ rowptr, uint32_t nv, uint32_t *__restrict__ deg) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        deg[v] = rowptr[v + 1] - rowptr[v];
}

/* Out-degrees as a histogram of the sources. Counts of ids below OUTDEG_WIN go
 * to per-block shared-memory counters first (the most-cited sources of power-law
 * graphs, R-MAT's among them, have small ids; this takes their contention off
 * the global atomics) and are added to the global counts once per block. */
constexpr uint32_t OUTDEG_WIN = 32768;
__global__ void __launch_bounds__(1024) k_outdeg_hist(const uint32_t *__restrict__ col, uint64_t n,
                                                      uint32_t win, uint32_t *__restrict__ outdeg) {
    extern __shared__ uint32_t s_cnt[];
    for (uint32_t i = threadIdx.x; i < win; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = col[i];
        if (u < win) atomicAdd(s_cnt + u, 1u);
        else atomicAdd(outdeg + u, 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < win; i += blockDim.x)
        if (s_cnt[i]) atomicAdd(outdeg + i, s_cnt[i]);
}

/* largest r in [0, nv) with rowptr[r] <= x (the non-empty row holding edge x);
 * called by a whole warp: 32 probes per step, about log32(nv) dependent loads */
__device__ uint32_t row_of(const uint32_t *rowptr, uint32_t nv, uint32_t x) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo = 0, hi = nv; /* answer in [lo, hi) */
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t probe = lo + lane * step; /* probe 0 is lo itself, and rowptr[lo] <= x */
        const bool ok = probe < hi && rowptr[probe] <= x;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok) | 1u;
        const uint32_t nlo = lo + (31u - __clz(m)) * step; /* the largest probe <= x */
        hi = nlo + step < hi ? nlo + step : hi;
        lo = nlo;
    }
    return lo;
}

/* One warp: the k-way merge sink's interval cuts (sharder.hpp:861-892, :962).
 * Every lane follows the same cuts (the searches are warp-wide); lane 0 writes. */
__global__ void k_intervals(const uint32_t *__restrict__ rowptr, uint32_t nv, uint32_t P, uint32_t *last,
                            uint32_t *count) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const bool lead = threadIdx.x == 0;
    const uint64_t E = rowptr[nv];
    const uint32_t max_vid = nv - 1;
    if (E == 0 || P <= 1) {
        if (lead) {
            last[0] = max_vid;
            *count = 1;
        }
        return;
    }
    uint64_t eps = E / P + 1, base = 0;
    uint32_t shard = 0;
    while (shard < P - 1) {
        uint64_t target = base + (eps > 0 ? eps : 1);
        if (target >= E) break;
        uint32_t r = row_of(rowptr, nv, (uint32_t)target);
        uint64_t j = (rowptr[r] == target) ? target : (uint64_t)rowptr[r + 1];
        if (j >= E) break;
        const uint32_t cut = row_of(rowptr, nv, (uint32_t)(j - 1));
        if (lead) last[shard] = cut;
        ++shard;
        eps = (E - j) / (P - shard);
        base = j;
    }
    const uint32_t fin = (shard == P - 1) ? max_vid : row_of(rowptr, nv, (uint32_t)(E - 1));
    if (lead) {
        last[shard] = fin;
        *count = shard + 1;
    }
}

}  // namespace

unsigned grid_for(uint64_t n, int threads = 256);

int unique_u64(const uint64_t *in, uint64_t n, uint32_t *flags, uint32_t *total_dev, uint64_t *out, cudaStream_t s) {
    if (n == 0) {
        GCG_CUDA(cudaMemsetAsync(total_dev, 0, 4, s));
        return GCG_OK;
    }
    k_unique_flags<<<grid_for(n), 256, 0, s>>>(in, n, flags);
    GCG_LAUNCH_CHECK();
    GCG_TRY(scan_u32(flags, flags, n, total_dev, s));
    k_unique_scatter<<<grid_for(n), 256, 0, s>>>(in, n, flags, out);
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

int csr_from_sorted_keys(const uint64_t *keys, uint64_t n, uint32_t vbits, uint32_t nrows, uint32_t *rowptr,
                         uint32_t *col, cudaStream_t s) {
    if (n == 0) {
        GCG_CUDA(cudaMemsetAsync(rowptr, 0, ((size_t)nrows + 1) * 4, s));
        return GCG_OK;
    }
    k_csr_from_keys<<<grid_for(std::max<uint64_t>(n, (uint64_t)nrows + 1)), 256, 0, s>>>(keys, n, vbits, nrows, rowptr,
                                                                                       col);
    GCG_LAUNCH_CHECK();
    return GCG_OK;
}

unsigned grid_for(uint64_t n, int threads) {
    uint64_t b = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)num_sms() * 32;
    if (b > cap) b = cap;
    if (b == 0) b = 1;
    return (unsigned)b;
}

namespace {

constexpr uint64_t PIPE_MIN_EDGES = 1ull << 24;
constexpr int PIPE_CHUNKS = 16; /* a power of two: runs merge in equal pairs */

uint32_t id_bits(uint32_t maxid) {
    uint32_t b = 1;
    while (b < 32 && (1ull << b) <= maxid) ++b;
    return b;
}

/* Host edge arrays, sorted while they cross PCIe. The edges are copied in
 * PIPE_CHUNKS pieces on a copy stream; each piece is scanned (self-loops, max
 * id, range) as soon as it lands; its keys (dst << 32 | src) are radix-sorted on
 * the sort stream while later pieces are still in flight (only the digits its
 * largest id needs) and merged at once into one run of all earlier pieces,
 * except the last piece, whose merge the caller fuses with the duplicate filter
 * and the CSR decode. After the last piece lands, only its sort remains. The
 * run of the earlier pieces occupies [0, len) of keys or tmp (the buffers swap
 * at every merge); a sorted piece is moved to that buffer at its own offset, so
 * a merge never writes over a run it reads. The two final runs come back in
 * run[0], run[1] (pointer, length; both in one buffer); the scan results of all
 * pieces are combined into *info. With outcnt, the raw out-degree of every id is
 * counted into outcnt (grown as larger ids arrive; outgrown buffers are kept in
 * old). */
struct SortedRuns {
    const uint64_t *p[2];
    uint64_t n[2];
};

int sort_host_edges(const uint32_t *src_u, const uint32_t *dst_u, uint64_t m, bool sym, uint32_t nv_given,
                    uint32_t *sbuf, uint32_t *dbuf_, uint64_t *keys, uint64_t *tmp, SortedRuns *runs,
                    ScanInfo *info, dbuf<uint32_t> *outcnt, std::vector<dbuf<uint32_t> *> &old) {
    const int K = PIPE_CHUNKS;
    const uint64_t cm = ((m + K - 1) / K + 4095) & ~(uint64_t)4095;
    const uint64_t kmul = sym ? 2 : 1;
    cudaStream_t cs = nullptr, ss = nullptr, ks = nullptr;
    cudaEvent_t ev_copy[PIPE_CHUNKS] = {}, ev_scan[PIPE_CHUNKS] = {};
    ScanInfo *h_info = nullptr;
    tbuf<ScanInfo> d_info;
    int st = GCG_OK;
    auto done = [&](int status) {
        if (ks) cudaStreamSynchronize(ks);
        if (ss) cudaStreamSynchronize(ss);
        if (cs) cudaStreamSynchronize(cs);
        for (int i = 0; i < K; ++i) {
            if (ev_copy[i]) cudaEventDestroy(ev_copy[i]);
            if (ev_scan[i]) cudaEventDestroy(ev_scan[i]);
        }
        if (cs) cudaStreamDestroy(cs);
        if (ss) cudaStreamDestroy(ss);
        if (ks) cudaStreamDestroy(ks);
        if (h_info) host_free(h_info);
        return status;
    };
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking) != cudaSuccess)
        return done(fail(GCG_ERR_CUDA, "edge pipeline: stream creation failed"));
    for (int i = 0; i < K; ++i)
        if (cudaEventCreateWithFlags(&ev_copy[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_scan[i], cudaEventDisableTiming) != cudaSuccess)
            return done(fail(GCG_ERR_CUDA, "edge pipeline: event creation failed"));
    if (host_alloc((void **)&h_info, sizeof(ScanInfo) * K) != cudaSuccess)
        return done(fail(GCG_ERR_NOMEM, "edge pipeline: pinned scan results"));
    if ((st = d_info.alloc(K, 0))) return done(st);
    if (cudaMemsetAsync(d_info.get(), 0, sizeof(ScanInfo) * K, 0) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess) /* the buffers exist before the other streams use them */
        return done(fail(GCG_ERR_CUDA, "edge pipeline: setup"));

    /* every piece's copy and scan are queued at once; the copies run back to back */
    for (int i = 0; i < K; ++i) {
        const uint64_t c0 = (uint64_t)i * cm, cn = std::min<uint64_t>(cm, m - std::min(m, c0));
        if (cn) {
            if (cudaMemcpyAsync(sbuf + c0, src_u + c0, cn * 4, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
                cudaMemcpyAsync(dbuf_ + c0, dst_u + c0, cn * 4, cudaMemcpyHostToDevice, cs) != cudaSuccess)
                return done(fail(GCG_ERR_CUDA, "edge pipeline: host to device copy"));
        }
        cudaEventRecord(ev_copy[i], cs);
        cudaStreamWaitEvent(ss, ev_copy[i], 0);
        if (cn) k_scan_edges<<<grid_for(cn), 256, 0, ss>>>(sbuf + c0, dbuf_ + c0, cn, nv_given, d_info.get() + i);
        cudaMemcpyAsync(h_info + i, d_info.get() + i, sizeof(ScanInfo), cudaMemcpyDeviceToHost, ss);
        cudaEventRecord(ev_scan[i], ss);
    }
    if (cudaGetLastError() != cudaSuccess) return done(fail(GCG_ERR_CUDA, "edge pipeline: queueing failed"));

    uint64_t *acc = keys; /* buffer of the run of the earlier pieces, at [0, acc_len) */
    uint64_t acc_len = 0;
    info->kept = 0;
    info->maxid = 0;
    info->bad = 0;
    for (int i = 0; i < K; ++i) {
        if (cudaEventSynchronize(ev_scan[i]) != cudaSuccess)
            return done(fail(GCG_ERR_CUDA, "edge pipeline: copy or scan failed"));
        const ScanInfo ci = h_info[i];
        info->kept += ci.kept;
        info->maxid = std::max(info->maxid, ci.maxid);
        info->bad |= ci.bad;
        const uint64_t c0 = (uint64_t)i * cm, cn = std::min<uint64_t>(cm, m - std::min(m, c0));
        const uint64_t k0 = kmul * c0, kn = kmul * cn;
        cudaStreamWaitEvent(ks, ev_scan[i], 0);
        if (outcnt && !info->bad && (uint64_t)info->maxid + 1 > outcnt->n) {
            uint64_t cap = (uint64_t)1 << 16;
            while (cap < (uint64_t)info->maxid + 1) cap <<= 1;
            dbuf<uint32_t> *grown = new dbuf<uint32_t>();
            if (grown->alloc(cap)) {
                delete grown;
                return done(GCG_ERR_NOMEM);
            }
            if (cudaMemsetAsync(grown->get(), 0, cap * 4, ks) != cudaSuccess ||
                (outcnt->n && cudaMemcpyAsync(grown->get(), outcnt->get(), outcnt->n * 4, cudaMemcpyDeviceToDevice,
                                              ks) != cudaSuccess)) {
                delete grown;
                return done(fail(GCG_ERR_CUDA, "edge pipeline: out-degree counts"));
            }
            /* the outgrown buffer may still be read by queued work: freed with the build */
            dbuf<uint32_t> *prev = new dbuf<uint32_t>();
            std::swap(prev->p, outcnt->p);
            std::swap(prev->n, outcnt->n);
            std::swap(outcnt->p, grown->p);
            std::swap(outcnt->n, grown->n);
            delete grown;
            old.push_back(prev);
        }
        if (kn) {
            k_make_keys<<<grid_for(cn), 256, 0, ks>>>(sbuf + c0, dbuf_ + c0, cn, 32, sym ? 1 : 0, keys + k0,
                                                      (outcnt && !info->bad) ? outcnt->get() : nullptr);
            const int cb = (int)id_bits(ci.maxid);
            uint64_t *r1 = nullptr, *r2 = nullptr;
            if ((st = radix_sort_u64(keys + k0, tmp + k0, kn, 0, cb, &r1, ks))) return done(st);
            uint64_t *o1 = (r1 == keys + k0) ? tmp + k0 : keys + k0;
            if ((st = radix_sort_u64(r1, o1, kn, 32, 32 + cb, &r2, ks))) return done(st);
            if (i == 0) acc = (r2 == keys + k0) ? keys : tmp; /* the first run stays where it was sorted */
            if (r2 != acc + k0 && cudaMemcpyAsync(acc + k0, r2, kn * 8, cudaMemcpyDeviceToDevice, ks) != cudaSuccess)
                return done(fail(GCG_ERR_CUDA, "edge pipeline: run copy"));
        }
        if (i == 0 || i == K - 1) {
            if (i == 0) acc_len = kn;
            continue; /* the last piece's merge is the caller's */
        }
        if (kn) {
            uint64_t *to = (acc == keys) ? tmp : keys;
            if ((st = merge_u64(acc, acc_len, acc + k0, kn, to, ks))) return done(st);
            acc = to;
            acc_len += kn;
        }
    }
    const uint64_t kl = kmul * std::min<uint64_t>(m, (uint64_t)(K - 1) * cm); /* the last piece's offset */
    if (acc_len != kl) return done(fail(GCG_ERR_CUDA, "edge pipeline: runs left unmerged"));
    runs->p[0] = acc;
    runs->n[0] = acc_len;
    runs->p[1] = acc + kl;
    runs->n[1] = kmul * m - kl;
    if (cudaStreamSynchronize(ks) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return done(fail(GCG_ERR_CUDA, std::string("edge pipeline: ") + cudaGetErrorString(cudaGetLastError())));
    return done(GCG_OK);
}

int build_graph(const uint32_t *src_u, const uint32_t *dst_u, uint64_t m, uint32_t nv_given, uint32_t flags,
                uint32_t nshards, gcg_graph **out) {
    cudaStream_t s = 0;
    const bool sym = (flags & GCG_BUILD_SYMMETRISE) != 0;
    const uint64_t nk = sym ? 2 * m : m;
    tbuf<uint32_t> sbuf, dbuf_;
    tbuf<uint64_t> keys, tmp;
    uint64_t *sorted = nullptr;
    SortedRuns runs = {{nullptr, nullptr}, {0, 0}};
    ScanInfo info;
    uint32_t kbits = 0; /* width of the src half of a key: 32 when sorted in pieces, else vbits */
    const bool pipelined = m >= PIPE_MIN_EDGES && !is_device_ptr(src_u) && !is_device_ptr(dst_u);
    const bool want_out = !(flags & GCG_BUILD_NO_OUT_CSR);
    dbuf<uint32_t> outcnt; /* raw out-degrees counted while the pieces are sorted */
    std::vector<dbuf<uint32_t> *> outgrown;
    struct FreeOld {
        std::vector<dbuf<uint32_t> *> &v;
        ~FreeOld() {
            for (auto *b : v) delete b;
        }
    } free_old{outgrown};
    const uint32_t *src = src_u, *dst = dst_u;
    if (pipelined) {
        if (sbuf.alloc(m, s) || dbuf_.alloc(m, s) || keys.alloc(nk, s) || tmp.alloc(nk, s)) return GCG_ERR_NOMEM;
        GCG_TRY(sort_host_edges(src_u, dst_u, m, sym, nv_given, sbuf.get(), dbuf_.get(), keys.get(), tmp.get(),
                                &runs, &info, want_out ? nullptr : &outcnt, outgrown));
        kbits = 32;
    } else {
        /* stage inputs */
        if (m > 0 && !is_device_ptr(src_u)) {
            GCG_TRY(sbuf.alloc(m, s));
            GCG_TRY(copy_in(sbuf.get(), src_u, m * 4, s));
            src = sbuf.get();
        }
        if (m > 0 && !is_device_ptr(dst_u)) {
            GCG_TRY(dbuf_.alloc(m, s));
            GCG_TRY(copy_in(dbuf_.get(), dst_u, m * 4, s));
            dst = dbuf_.get();
        }
        /* max id, kept count, range check */
        tbuf<ScanInfo> d_info;
        GCG_TRY(d_info.alloc(1, s));
        GCG_CUDA(cudaMemsetAsync(d_info.get(), 0, sizeof(ScanInfo), s));
        if (m > 0) {
            k_scan_edges<<<grid_for(m), 256, 0, s>>>(src, dst, m, nv_given, d_info.get());
            GCG_LAUNCH_CHECK();
        }
        GCG_CUDA(cudaMemcpyAsync(&info, d_info.get(), sizeof(info), cudaMemcpyDeviceToHost, s));
        GCG_CUDA(cudaStreamSynchronize(s));
    }
    if (info.bad) return fail(GCG_ERR_INVALID, "gcg_graph_from_edges: vertex id >= num_vertices");
    const uint64_t nv64 = nv_given ? (uint64_t)nv_given : (uint64_t)info.maxid + 1; /* sharder.hpp:925 */
    if (nv64 > MAX_VERTICES)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_from_edges: " + std::to_string(nv64) +
                                             " vertices; at most 2^32 - 2^26 (largest id 4227858431)");
    const uint32_t nv = (uint32_t)nv64;
    const uint64_t kept = sym ? 2 * (uint64_t)info.kept : (uint64_t)info.kept;
    if (kept > MAX_EDGES)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_from_edges: more than 2^32 - 2^26 edges after filtering");
    uint32_t vbits = 1;
    while (vbits < 32 && (1ull << vbits) < nv) ++vbits;
    if (!pipelined) kbits = vbits;

    gcg_graph *g = new gcg_graph();
    g->nv = nv;
    g->vbits = vbits;
    g->symmetric = sym;
    g->build_flags = flags;
    g->nshards_req = nshards ? nshards : 1;
    g->stream = s;
    auto cleanup = [&](int st) {
        delete g;
        return st;
    };

    uint64_t ne = 0;
    if (g->in_rowptr.alloc((size_t)nv + 1) || g->in_col.alloc(kept) || g->indeg.alloc(nv) || g->outdeg.alloc(nv))
        return cleanup(GCG_ERR_NOMEM);
    {
        int st = GCG_OK;
        if (!pipelined && nk > 0) {
            if (keys.alloc(nk, s) || tmp.alloc(nk, s)) return cleanup(GCG_ERR_NOMEM);
            k_make_keys<<<grid_for(m), 256, 0, s>>>(src, dst, m, vbits, sym ? 1 : 0, keys.get(), nullptr);
            if (cudaGetLastError() != cudaSuccess) return cleanup(fail(GCG_ERR_CUDA, "k_make_keys launch"));
            st = radix_sort_u64(keys.get(), tmp.get(), nk, 0, 2 * (int)vbits, &sorted, s);
            if (st) return cleanup(st);
            runs.p[0] = sorted;
            runs.n[0] = nk;
        }
        /* the kept keys go to the buffer that holds no run, when the out-CSR needs them */
        uint64_t *kept_keys = nullptr;
        if (want_out && kept > 0) kept_keys = (runs.p[0] >= keys.get() && runs.p[0] < keys.get() + nk) ? tmp.get()
                                                                                                      : keys.get();
        st = merge_unique_csr(runs.p[0], runs.n[0], runs.p[1], runs.n[1], kept, (flags & GCG_BUILD_DEDUP) != 0,
                              kbits, nv, g->in_rowptr.get(), g->in_col.get(), kept_keys,
                              outcnt.get() && !want_out ? outcnt.get() : nullptr, &ne, s);
        if (st) return cleanup(st);
        sorted = kept_keys;
    }
    g->ne = ne;
    k_degree<<<grid_for(nv), 256, 0, s>>>(g->in_rowptr.get(), nv, g->indeg.get());
    if (want_out) {
        if (g->out_rowptr.alloc((size_t)nv + 1) || g->out_col.alloc(ne)) return cleanup(GCG_ERR_NOMEM);
        if (ne == 0) {
            cudaMemsetAsync(g->out_rowptr.get(), 0, ((size_t)nv + 1) * 4, s);
        } else {
            uint64_t *a = (sorted == keys.get()) ? tmp.get() : keys.get();
            uint64_t *b = sorted;
            k_swap_key<<<grid_for(ne), 256, 0, s>>>(sorted, ne, kbits, a);
            uint64_t *res = nullptr;
            /* stable sort by the source half only: (dst, src) order -> (src, dst) */
            int st = radix_sort_u64(a, b, ne, (int)kbits, (int)(kbits + vbits), &res, s);
            if (st) return cleanup(st);
            k_csr_from_keys<<<grid_for(ne), 256, 0, s>>>(res, ne, kbits, nv, g->out_rowptr.get(), g->out_col.get());
        }
        k_degree<<<grid_for(nv), 256, 0, s>>>(g->out_rowptr.get(), nv, g->outdeg.get());
        g->has_out = true;
    } else if (outcnt.get()) {
        /* counted during the piecewise sort, repeats taken off by the finish; ids
         * above the largest one seen (a caller-given vertex count) have none */
        const size_t have = std::min<size_t>(nv, outcnt.n);
        if (have < nv) cudaMemsetAsync(g->outdeg.get() + have, 0, (nv - have) * 4, s);
        cudaMemcpyAsync(g->outdeg.get(), outcnt.get(), have * 4, cudaMemcpyDeviceToDevice, s);
    } else {
        cudaMemsetAsync(g->outdeg.get(), 0, (size_t)nv * 4, s);
        if (ne > 0) {
            /* sources are the low halves of the sorted keys; take them from in_col */
            const uint32_t win = std::min<uint32_t>(nv, OUTDEG_WIN);
            static bool attr = false;
            if (!attr) {
                cudaFuncSetAttribute(k_outdeg_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(OUTDEG_WIN * 4));
                attr = true;
            }
            k_outdeg_hist<<<num_sms(), 1024, (size_t)win * 4, s>>>(g->in_col.get(), ne, win, g->outdeg.get());
        }
    }
    /* intervals */
    uint32_t P = nshards ? nshards : 1;
    tbuf<uint32_t> d_count;
    if (g->intervals_dev.alloc(P) || d_count.alloc(1, s)) return cleanup(GCG_ERR_NOMEM);
    k_intervals<<<1, 32, 0, s>>>(g->in_rowptr.get(), nv, P, g->intervals_dev.get(), d_count.get());
    if (cudaGetLastError() != cudaSuccess) return cleanup(fail(GCG_ERR_CUDA, "graph build kernels failed to launch"));
    uint32_t cnt = 0;
    g->intervals_host = (uint32_t *)malloc((size_t)P * 4);
    if (cudaMemcpyAsync(&cnt, d_count.get(), 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(g->intervals_host, g->intervals_dev.get(), (size_t)P * 4, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return cleanup(fail(GCG_ERR_CUDA, std::string("graph build failed: ") + cudaGetErrorString(cudaGetLastError())));
    g->nshards = cnt;
    *out = g;
    return GCG_OK;
}

}  // namespace
namespace {

/* ---- edge updates (dynamic graphs) ------------------------------------------ */

/* every edge of the in-CSR as (src, dst): a warp per row */
__global__ void k_edges_of(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                           uint32_t *__restrict__ src, uint32_t *__restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31u, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarps)
        for (uint32_t i = rowptr[v] + lane; i < rowptr[v + 1]; i += 32u) {
            src[i] = col[i];
            dst[i] = v;
        }
}

/* the added edges after the existing ones; both directions for a symmetric graph */
__global__ void k_append_edges(const uint32_t *__restrict__ s, const uint32_t *__restrict__ d, uint64_t m, int both,
                               uint64_t off, uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                               uint32_t *__restrict__ maxid) {
    uint32_t mx = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = s[i], b = d[i];
        src[off + i] = a;
        dst[off + i] = b;
        if (both) {
            src[off + m + i] = b;
            dst[off + m + i] = a;
        }
        mx = max(mx, max(a, b));
    }
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(maxid, mx);
}

/* keys (dst << vbits | src) of the edges to delete; ids outside the graph can
 * match nothing and become the all-ones key */
__global__ void k_delete_keys(const uint32_t *__restrict__ s, const uint32_t *__restrict__ d, uint64_t m, int both,
                              uint32_t nv, uint32_t vbits, uint64_t *__restrict__ keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = s[i], b = d[i];
        const bool ok = a < nv && b < nv;
        keys[i] = ok ? (((uint64_t)b << vbits) | a) : ~0ull;
        if (both) keys[m + i] = ok ? (((uint64_t)a << vbits) | b) : ~0ull;
    }
}

/* keep[i] = 1 unless edge i's key is in the sorted delete list */
__global__ void k_keep_flags(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                             const uint64_t *__restrict__ del, uint64_t nd, uint32_t vbits, uint32_t *__restrict__ keep) {
    const uint32_t lane = threadIdx.x & 31u, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarps)
        for (uint32_t i = rowptr[v] + lane; i < rowptr[v + 1]; i += 32u) {
            const uint64_t key = ((uint64_t)v << vbits) | col[i];
            uint64_t lo = 0, hi = nd;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (del[mid] < key) lo = mid + 1; else hi = mid;
            }
            keep[i] = (lo < nd && del[lo] == key) ? 0u : 1u;
        }
}

__global__ void k_compact_edges(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ col, uint32_t nv,
                                const uint32_t *__restrict__ keep, const uint32_t *__restrict__ pos,
                                uint32_t *__restrict__ src, uint32_t *__restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31u, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarps)
        for (uint32_t i = rowptr[v] + lane; i < rowptr[v + 1]; i += 32u)
            if (keep[i]) {
                src[pos[i]] = col[i];
                dst[pos[i]] = v;
            }
}

/* g takes over ng's arrays, plans and sizes (its handle and stream stay); ng
 * leaves with g's old ones and is deleted by the caller */
void swap_graph(gcg_graph *g, gcg_graph *ng) {
    std::swap(g->nv, ng->nv);
    std::swap(g->ne, ng->ne);
    std::swap(g->nshards, ng->nshards);
    std::swap(g->vbits, ng->vbits);
    auto sw = [](dbuf<uint32_t> &a, dbuf<uint32_t> &b) {
        std::swap(a.p, b.p);
        std::swap(a.n, b.n);
    };
    sw(g->in_rowptr, ng->in_rowptr);
    sw(g->in_col, ng->in_col);
    sw(g->out_rowptr, ng->out_rowptr);
    sw(g->out_col, ng->out_col);
    sw(g->indeg, ng->indeg);
    sw(g->outdeg, ng->outdeg);
    sw(g->intervals_dev, ng->intervals_dev);
    std::swap(g->has_out, ng->has_out);
    std::swap(g->intervals_host, ng->intervals_host);
    std::swap(g->plan, ng->plan);
    std::swap(g->cplan, ng->cplan);
    std::swap(g->pplan, ng->pplan);
    std::swap(g->gsplan, ng->gsplan);
}

int rebuild_from(gcg_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t nv) {
    if (m > 0xFFFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "edge update: more than 2^32-1 edges");
    gcg_graph *ng = nullptr;
    /* the edge list already holds both directions of a symmetric graph */
    GCG_TRY(build_graph(src, dst, m, nv, g->build_flags & ~GCG_BUILD_SYMMETRISE, g->nshards_req, &ng));
    cudaStreamSynchronize(g->stream);
    swap_graph(g, ng);
    delete ng; /* the old arrays and the plans built for them */
    return GCG_OK;
}

int add_edges(gcg_graph *g, const uint32_t *s_u, const uint32_t *d_u, uint64_t m) {
    cudaStream_t s = 0;
    GCG_CUDA(cudaStreamSynchronize(g->stream));
    tbuf<uint32_t> sb, db, src, dst, mx;
    const uint32_t *sa = s_u, *da = d_u;
    if (m > 0 && !is_device_ptr(s_u)) {
        GCG_TRY(sb.alloc(m, s));
        GCG_TRY(copy_in(sb.get(), s_u, m * 4, s));
        sa = sb.get();
    }
    if (m > 0 && !is_device_ptr(d_u)) {
        GCG_TRY(db.alloc(m, s));
        GCG_TRY(copy_in(db.get(), d_u, m * 4, s));
        da = db.get();
    }
    const int both = g->symmetric ? 1 : 0;
    const uint64_t total = g->ne + (both ? 2 * m : m);
    if (total > MAX_EDGES) return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_add_edges: more than 2^32 - 2^26 edges");
    GCG_TRY(src.alloc(std::max<uint64_t>(total, 1), s));
    GCG_TRY(dst.alloc(std::max<uint64_t>(total, 1), s));
    GCG_TRY(mx.alloc(1, s));
    GCG_CUDA(cudaMemsetAsync(mx.get(), 0, 4, s));
    if (g->ne) k_edges_of<<<grid_for((uint64_t)g->nv * 32), 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), g->nv,
                                                                         src.get(), dst.get());
    if (m) k_append_edges<<<grid_for(m), 256, 0, s>>>(sa, da, m, both, g->ne, src.get(), dst.get(), mx.get());
    GCG_LAUNCH_CHECK();
    uint32_t maxid = 0;
    GCG_CUDA(cudaMemcpyAsync(&maxid, mx.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    const uint64_t nv = std::max<uint64_t>(g->nv, m ? (uint64_t)maxid + 1 : 0);
    if (nv > MAX_VERTICES) return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_add_edges: vertex ids at most 2^32 - 2^26 - 1");
    return rebuild_from(g, src.get(), dst.get(), total, (uint32_t)nv);
}

int delete_edges(gcg_graph *g, const uint32_t *s_u, const uint32_t *d_u, uint64_t m) {
    cudaStream_t s = 0;
    GCG_CUDA(cudaStreamSynchronize(g->stream));
    if (m == 0 || g->ne == 0) return GCG_OK;
    tbuf<uint32_t> sb, db, keep, src, dst, total;
    tbuf<uint64_t> keys, tmp;
    const uint32_t *sa = s_u, *da = d_u;
    if (!is_device_ptr(s_u)) {
        GCG_TRY(sb.alloc(m, s));
        GCG_TRY(copy_in(sb.get(), s_u, m * 4, s));
        sa = sb.get();
    }
    if (!is_device_ptr(d_u)) {
        GCG_TRY(db.alloc(m, s));
        GCG_TRY(copy_in(db.get(), d_u, m * 4, s));
        da = db.get();
    }
    const int both = g->symmetric ? 1 : 0;
    const uint64_t nd = both ? 2 * m : m;
    GCG_TRY(keys.alloc(nd, s));
    GCG_TRY(tmp.alloc(nd, s));
    k_delete_keys<<<grid_for(m), 256, 0, s>>>(sa, da, m, both, g->nv, g->vbits, keys.get());
    GCG_LAUNCH_CHECK();
    uint64_t *sorted = nullptr;
    GCG_TRY(radix_sort_u64(keys.get(), tmp.get(), nd, 0, 64, &sorted, s));
    const uint64_t ne = g->ne;
    GCG_TRY(keep.alloc(ne, s));
    GCG_TRY(total.alloc(1, s));
    const unsigned wb = grid_for((uint64_t)g->nv * 32);
    k_keep_flags<<<wb, 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), g->nv, sorted, nd, g->vbits, keep.get());
    GCG_LAUNCH_CHECK();
    tbuf<uint32_t> pos;
    GCG_TRY(pos.alloc(ne, s));
    GCG_TRY(scan_u32(keep.get(), pos.get(), ne, total.get(), s));
    uint32_t kept = 0;
    GCG_CUDA(cudaMemcpyAsync(&kept, total.get(), 4, cudaMemcpyDeviceToHost, s));
    GCG_CUDA(cudaStreamSynchronize(s));
    if (kept == ne) return GCG_OK; /* nothing listed was present */
    GCG_TRY(src.alloc(std::max<uint32_t>(kept, 1), s));
    GCG_TRY(dst.alloc(std::max<uint32_t>(kept, 1), s));
    k_compact_edges<<<wb, 256, 0, s>>>(g->in_rowptr.get(), g->in_col.get(), g->nv, keep.get(), pos.get(), src.get(),
                                       dst.get());
    GCG_LAUNCH_CHECK();
    return rebuild_from(g, src.get(), dst.get(), kept, g->nv);
}

}  // namespace

}  // namespace gcg

using namespace gcg;

extern "C" {

int gcg_graph_add_edges(gcg_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t m) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_graph_add_edges: null graph");
    if (m > 0 && (!src || !dst)) return fail(GCG_ERR_INVALID, "gcg_graph_add_edges: null edge arrays");
    return add_edges(g, src, dst, m);
}

int gcg_graph_delete_edges(gcg_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t m) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_graph_delete_edges: null graph");
    if (m > 0 && (!src || !dst)) return fail(GCG_ERR_INVALID, "gcg_graph_delete_edges: null edge arrays");
    return delete_edges(g, src, dst, m);
}

int gcg_graph_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t num_vertices,
                         uint32_t flags, uint32_t nshards, gcg_graph **out) {
    if (!out) return fail(GCG_ERR_INVALID, "gcg_graph_from_edges: null out");
    *out = nullptr;
    if (m > 0 && (!src || !dst)) return fail(GCG_ERR_INVALID, "gcg_graph_from_edges: null edge arrays");
    if (m > 0xFFFFFFFFull) return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_from_edges: more than 2^32-1 edges");
    if (num_vertices > MAX_VERTICES)
        return fail(GCG_ERR_UNSUPPORTED, "gcg_graph_from_edges: num_vertices above 2^32 - 2^26");
    return build_graph(src, dst, m, num_vertices, flags, nshards, out);
}

int gcg_graph_intervals(const gcg_graph *g, uint32_t *last_vid) {
    if (!g || !last_vid) return fail(GCG_ERR_INVALID, "gcg_graph_intervals: null argument");
    GCG_CUDA(cudaMemcpy(last_vid, g->intervals_host, (size_t)g->nshards * 4, cudaMemcpyDefault));
    return GCG_OK;
}

}  // extern "C"

namespace gcg {
namespace {
__global__ void k_interleave_deg(const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ outdeg, uint32_t nv,
                                 int32_t *__restrict__ pairs) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        pairs[2 * (size_t)v] = (int32_t)indeg[v];
        pairs[2 * (size_t)v + 1] = (int32_t)outdeg[v];
    }
}
}  // namespace
}  // namespace gcg

extern "C" {

int gcg_graph_degrees(const gcg_graph *g, int32_t *pairs) {
    if (!g || !pairs) return fail(GCG_ERR_INVALID, "gcg_graph_degrees: null argument");
    tbuf<int32_t> tmp;
    int32_t *dst = pairs;
    bool dev = is_device_ptr(pairs);
    if (!dev) {
        GCG_TRY(tmp.alloc((size_t)g->nv * 2, g->stream));
        dst = tmp.get();
    }
    k_interleave_deg<<<grid_for(g->nv), 256, 0, g->stream>>>(g->indeg.get(), g->outdeg.get(), g->nv, dst);
    GCG_LAUNCH_CHECK();
    if (!dev) GCG_TRY(copy_out(pairs, dst, (size_t)g->nv * 8, g->stream));
    else GCG_CUDA(cudaStreamSynchronize(g->stream));
    return GCG_OK;
}

int gcg_graph_csr(const gcg_graph *g, int which, uint32_t *rowptr, uint32_t *col) {
    if (!g) return fail(GCG_ERR_INVALID, "gcg_graph_csr: null graph");
    const uint32_t *rp, *cl;
    if (which == GCG_CSR_IN) {
        rp = g->in_rowptr.get();
        cl = g->in_col.get();
    } else if (which == GCG_CSR_OUT) {
        if (!g->has_out) return fail(GCG_ERR_INVALID, "gcg_graph_csr: graph built without the out-edge CSR");
        rp = g->out_rowptr.get();
        cl = g->out_col.get();
    } else {
        return fail(GCG_ERR_INVALID, "gcg_graph_csr: which must be GCG_CSR_IN or GCG_CSR_OUT");
    }
    if (rowptr) GCG_TRY(copy_out(rowptr, rp, ((size_t)g->nv + 1) * 4, g->stream));
    if (col) GCG_TRY(copy_out(col, cl, (size_t)g->ne * 4, g->stream));
    GCG_CUDA(cudaStreamSynchronize(g->stream));
    return GCG_OK;
}

int gcg_graph_write_metadata(const gcg_graph *g, const char *base) {
    if (!g || !base) return fail(GCG_ERR_INVALID, "gcg_graph_write_metadata: null argument");
    std::string b(base);
    /* <base>.<P>.intervals: one last-vid per line (sharder.hpp:909-920) */
    std::string fi = b + "." + std::to_string(g->nshards) + ".intervals";
    FILE *f = fopen(fi.c_str(), "w");
    if (!f) return fail(GCG_ERR_IO, "cannot write " + fi);
    for (uint32_t i = 0; i < g->nshards; ++i) fprintf(f, "%u\n", g->intervals_host[i]);
    fclose(f);
    /* <base>.numvertices (sharder.hpp:922-926) */
    std::string fn = b + ".numvertices";
    f = fopen(fn.c_str(), "w");
    if (!f) return fail(GCG_ERR_IO, "cannot write " + fn);
    fprintf(f, "%u\n", g->nv);
    fclose(f);
    /* <base>_degs.bin: struct degree {int in, out} per vertex (sharder.hpp:996-1006) */
    std::vector<int32_t> deg((size_t)g->nv * 2);
    GCG_TRY(gcg_graph_degrees(g, deg.data()));
    std::string fd = b + "_degs.bin";
    f = fopen(fd.c_str(), "wb");
    if (!f) return fail(GCG_ERR_IO, "cannot write " + fd);
    size_t w = fwrite(deg.data(), sizeof(int32_t), deg.size(), f);
    fclose(f);
    if (w != deg.size()) return fail(GCG_ERR_IO, "short write to " + fd);
    return GCG_OK;
}

}  // extern "C"
