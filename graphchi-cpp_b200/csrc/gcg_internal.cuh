/*
 * Internal declarations shared by the libgcgpu translation units.
 * Not part of the C ABI (that is include/gcgpu.h).
 */
#ifndef GCG_INTERNAL_CUH
#define GCG_INTERNAL_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "gcgpu.h"

namespace gcg {

/* ---- error handling: every exported entry point returns a gcg_status;
 *      the message of the last failure on this thread is kept. ---------- */
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);

#define GCG_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess) {                                                         \
            return ::gcg::fail(_e == cudaErrorMemoryAllocation ? GCG_ERR_NOMEM : GCG_ERR_CUDA, \
                               std::string(#call) + ": " + cudaGetErrorString(_e));      \
        }                                                                                \
    } while (0)

#define GCG_TRY(expr)                 \
    do {                              \
        int _s = (expr);              \
        if (_s != GCG_OK) return _s;  \
    } while (0)

#define GCG_LAUNCH_CHECK() GCG_CUDA(cudaGetLastError())

/* Largest vertex count and edge count (after filtering) of a graph, or of the union
 * of a batch: 2^32 - 2^26. Kernels index vertices, rows, chunks and edges with
 * 32-bit counters in grid-stride loops; no launch has more than 2^26 threads, so
 * below this bound no counter can step past 2^32 and wrap around. */
constexpr uint64_t MAX_VERTICES = (1ull << 32) - (1ull << 26);
constexpr uint64_t MAX_EDGES = (1ull << 32) - (1ull << 26);

/* ---- block cache (gcg_common.cu): freed device blocks and small pinned host
 *      blocks are kept per device and size class for the next allocation ---- */
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_free(void *p);
cudaError_t host_alloc(void **p, size_t bytes);
void host_free(void *p);
/* after an out-of-memory error: releases the current device's idle cached blocks
 * and the memory its default stream-ordered pool keeps */
void reclaim_device_memory();

/* ---- device buffers ----------------------------------------------------- */
template <typename T>
struct dbuf {
    T *p = nullptr;
    size_t n = 0;
    dbuf() = default;
    dbuf(const dbuf &) = delete;
    dbuf &operator=(const dbuf &) = delete;
    ~dbuf() { release(); }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = dev_alloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(GCG_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                            " bytes: " + cudaGetErrorString(e));
        }
        n = count;
        return GCG_OK;
    }
    void release() {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    T *get() const { return p; }
};

/* Keeps memory freed to the current device's default pool cached in this
 * process (release threshold = max), so repeated calls do not map and unmap
 * device memory at every synchronisation. Process-local; ends with the process. */
void pool_keep_memory();

/* Stream-ordered temporary buffer: allocated with cudaMallocAsync and released
 * with cudaFreeAsync on the same stream, so its lifetime follows the kernels
 * queued on that stream without host synchronisation. */
template <typename T>
struct tbuf {
    T *p = nullptr;
    cudaStream_t s = 0;
    tbuf() = default;
    tbuf(const tbuf &) = delete;
    tbuf &operator=(const tbuf &) = delete;
    ~tbuf() { release(); }
    int alloc(size_t count, cudaStream_t stream) {
        release();
        pool_keep_memory();
        s = stream;
        if (count == 0) count = 1;
        cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), stream);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            reclaim_device_memory();
            e = cudaMallocAsync((void **)&p, count * sizeof(T), stream);
        }
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(GCG_ERR_NOMEM, std::string("cudaMallocAsync of ") + std::to_string(count * sizeof(T)) +
                                            " bytes: " + cudaGetErrorString(e));
        }
        return GCG_OK;
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
    T *get() const { return p; }
};

/* Pointer classification: device-resident buffers are used in place; anything
 * else is treated as host memory and staged through a device copy. */
bool is_device_ptr(const void *p);

/* Copy count elements between a user pointer (host or device) and device memory. */
int copy_in(void *dst_dev, const void *src_user, size_t bytes, cudaStream_t s);
int copy_out(void *dst_user, const void *src_dev, size_t bytes, cudaStream_t s);

/* Number of SMs on the current device (cached). */
int num_sms();

/* ---- the graph handle: device-resident CSR blocks ---------------------- */
struct PrPlan;
struct ChunkPlan;
void free_chunk_plan(ChunkPlan *p);
struct PprPlan;
void free_ppr_plan(PprPlan *p);
struct GsPlan;
void free_gs_plan(GsPlan *p);

}  // namespace gcg

struct gcg_graph {
    uint32_t nv = 0;       /* vertices: max id + 1 (sharder.hpp:925) or caller-given */
    uint64_t ne = 0;       /* directed edges after filtering */
    uint32_t nshards = 0;  /* intervals produced */
    uint32_t vbits = 0;    /* bits of a vertex id (ceil log2 nv) */
    cudaStream_t stream = 0;

    /* in-edges grouped by destination, sources ascending (memory shard order) */
    gcg::dbuf<uint32_t> in_rowptr, in_col;
    /* out-edges grouped by source, destinations ascending (shard order by src) */
    gcg::dbuf<uint32_t> out_rowptr, out_col;
    bool has_out = false;
    bool symmetric = false; /* built with GCG_BUILD_SYMMETRISE: every in-list is the full neighbourhood */
    uint32_t build_flags = 0, nshards_req = 1; /* how it was built (edge updates rebuild the same way) */
    gcg::dbuf<uint32_t> indeg, outdeg;
    gcg::dbuf<uint32_t> intervals_dev; /* last vid per interval */
    uint32_t *intervals_host = nullptr;

    /* merge-path tiling of the in-CSR (CC, TC), built on first use */
    gcg::PrPlan *plan = nullptr;
    /* 256-edge chunk plan of the in-CSR (PageRank), built on first use */
    gcg::ChunkPlan *cplan = nullptr;
    /* row segments for batched personalised PageRank, built on first use */
    gcg::PprPlan *pplan = nullptr;
    /* level schedule of the exact Gauss-Seidel modes, built on first use */
    gcg::GsPlan *gsplan = nullptr;
    /* PageRank plan options of the many-graph union: it is one (each interval a
     * graph, whose rows must stay one contiguous range), and whether to relabel
     * its sources by out-degree within each interval (every graph keeps its own
     * id range) */
    bool union_of_graphs = false;
    bool relabel_per_interval = false;

    ~gcg_graph();
};

namespace gcg {

/* ---- radix sort (gcg_sort.cu) ------------------------------------------ */
/* Stable LSD sort of n 64-bit keys by bits [begin_bit, end_bit). keys and tmp
 * are device arrays of n; the sorted keys end in *result (keys or tmp). */
int radix_sort_u64(uint64_t *keys, uint64_t *tmp, uint64_t n, int begin_bit, int end_bit,
                   uint64_t **result, cudaStream_t s);

/* Exclusive scan of n uint32 values (device), returns the total through *total_dev
 * (device pointer, may be null). in and out may alias. */
int scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total_dev, cudaStream_t s);

/* Merge of sorted runs a[0..na) and b[0..nb) into out[0..na+nb), stable (a's
 * first on equal keys); out overlaps neither run. */
int merge_u64(const uint64_t *a, uint64_t na, const uint64_t *b, uint64_t nb, uint64_t *out, cudaStream_t s);

/* The sharder's last step in one pass: merges sorted runs a and b (b may be
 * null with nb = 0), keeps the first kept merged keys (the rest are self-loop
 * sentinels), drops repeats when dedup, and writes the CSR of the kept keys
 * (row = key >> kbits, column = low kbits): rowptr[0..nv], col[0..*ne). Also
 * writes the kept keys to keys_out and decrements outdeg_dup[column] for every
 * dropped repeat, when those are given. Synchronises s. */
int merge_unique_csr(const uint64_t *a, uint64_t na, const uint64_t *b, uint64_t nb, uint64_t kept, bool dedup,
                     uint32_t kbits, uint32_t nv, uint32_t *rowptr, uint32_t *col, uint64_t *keys_out,
                     uint32_t *outdeg_dup, uint64_t *ne, cudaStream_t s);

/* Unique of sorted keys: out[0..total) = distinct keys (flags: n scratch). */
int unique_u64(const uint64_t *in, uint64_t n, uint32_t *flags, uint32_t *total_dev, uint64_t *out, cudaStream_t s);

/* Sorted (row << vbits | col) keys -> CSR with nrows rows. */
int csr_from_sorted_keys(const uint64_t *keys, uint64_t n, uint32_t vbits, uint32_t nrows, uint32_t *rowptr,
                         uint32_t *col, cudaStream_t s);

/* ---- merge-path plan (gcg_plan.cu) ------------------------------------- */
struct PrPlan {
    uint32_t ntiles = 0;
    dbuf<uint32_t> tile_row, tile_edge; /* ntiles+1 merge-path coordinates */
};
int ensure_plan(gcg_graph *g);

/* exact Gauss-Seidel PageRank (gcg_pagerank_gs.cu) */
int pagerank_gs_exact(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats);

/* selective scheduling on a device frontier (gcg_frontier.cu) */
int pagerank_delta(gcg_graph *g, const gcg_pr_params *p, float *out_rank, gcg_pr_stats *stats);
int cc_label_propagation(gcg_graph *g, int scheduler, int max_iters, uint32_t *labels, gcg_cc_stats *stats,
                         int32_t *frontier_log);

constexpr int MP_THREADS = 256;
constexpr int MP_ITEMS = 8;
constexpr int MP_TILE = MP_THREADS * MP_ITEMS;

}  // namespace gcg

#endif
