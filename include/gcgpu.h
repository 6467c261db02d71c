/*
 * gcgpu — C ABI of the B200-native engine for GraphChi's parallel-sliding-windows
 * hot path: sharder -> graphchi_engine::run() -> GraphChiProgram::update() for
 * PageRank, connected components and triangle counting.
 *
 * Plain C types only: pointers, sizes, status codes. Every call returns a
 * gcg_status (0 = OK, negative = error) and never aborts; gcg_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * Pointer arguments marked "host or device" may point to host memory (pageable
 * or pinned) or to device memory of the current CUDA device; device memory is
 * used in place, host memory is staged through device copies on the graph's
 * stream. All work of a graph runs on its stream (gcg_graph_set_stream).
 * Calls on one graph handle are not thread-safe; distinct handles are.
 *
 * Each entry point cites the reference interface it replaces
 * (paths relative to the graphchi-cpp source tree).
 */
#ifndef GCGPU_H
#define GCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GCG_OK = 0,
    GCG_ERR_INVALID = -1,     /* bad argument (null, out of range, vertex id >= nv) */
    GCG_ERR_CUDA = -2,        /* CUDA runtime error (no device, launch failure) */
    GCG_ERR_NOMEM = -3,       /* device allocation failed */
    GCG_ERR_IO = -4,          /* file could not be read or written */
    GCG_ERR_FORMAT = -5,      /* malformed edge-list line */
    GCG_ERR_UNSUPPORTED = -6, /* request outside this build's limits */
    GCG_ERR_TIMEOUT = -7      /* a bounded device wait ran out */
} gcg_status;

typedef struct gcg_graph gcg_graph;

/* ---- graph construction: the device sharder ---------------------------- */

#define GCG_BUILD_DEDUP 0x1u      /* keep one copy of repeated (src,dst) */
#define GCG_BUILD_SYMMETRISE 0x2u /* add (dst,src) for every (src,dst) before dedup */
#define GCG_BUILD_NO_OUT_CSR 0x4u /* skip the src-grouped (out-edge) CSR */

/* Replaces sharder<ET>::preprocessing_add_edge + execute_sharding
 * (src/preprocessing/sharder.hpp:427-446, :535-548, :861-1008) for an edge list
 * already in memory. Self-loops are dropped (sharder.hpp:428-431). Builds, in
 * HBM: the in-edge CSR grouped by destination with sources ascending (what each
 * memory shard holds, memoryshard.hpp:384-519), the out-edge CSR grouped by
 * source with destinations ascending (each shard's src-sorted order,
 * sharder.hpp:640), in/out degrees (sharder.hpp:748-751) and `nshards` vertex
 * intervals split exactly like the sharder's k-way merge sink
 * (sharder.hpp:861-892). num_vertices = 0 means max id + 1 (sharder.hpp:925);
 * otherwise every id must be < num_vertices. nshards = 0 means 1.
 * src/dst: m entries each, host or device. Limits: m < 2^32; at most 2^32 - 2^26
 * vertices (ids up to 4227858431) and 2^32 - 2^26 edges after filtering, else
 * GCG_ERR_UNSUPPORTED. */
int gcg_graph_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t m,
                         uint32_t num_vertices, uint32_t flags, uint32_t nshards,
                         gcg_graph **out);

/* Replaces convert_edgelist (src/preprocessing/conversions.hpp:210-288) followed
 * by the sharder: parses a text edge list ("src<ws|,>dst[ value]" per line,
 * '#'/'%' comment lines, delimiters "\t, ", decimal ids), then builds the graph
 * as gcg_graph_from_edges. Parsing is multithreaded on the host. */
int gcg_graph_from_edgelist_file(const char *path, uint32_t flags, uint32_t nshards,
                                 gcg_graph **out);

/* Parses a text edge list into caller arrays without building a graph.
 * With src/dst NULL only counts: *m_out receives the number of edge lines. */
int gcg_parse_edgelist_file(const char *path, uint32_t *src, uint32_t *dst, uint64_t capacity,
                            uint64_t *m_out);

/* Frees the graph. Its device blocks go back to the library's block cache
 * (below), not to the driver. */
int gcg_graph_free(gcg_graph *g);

/* The library keeps freed device blocks (and small pinned host blocks) per device
 * and size class and hands them to later allocations of the same class, so a loop
 * that builds, solves and frees graphs calls neither cudaMalloc nor cudaFree after
 * its first pass. The reference allocates with malloc/free per run (no
 * counterpart). Freeing a block into the cache synchronises its device first, as
 * cudaFree does. The idle cache is capped per device by the environment variable
 * GCG_DEVICE_CACHE_MB (default: a quarter of the device's memory; 0 turns caching
 * off; host: GCG_HOST_CACHE_MB, default 256) and is emptied, and the allocation
 * retried, when the driver runs out of memory.
 * gcg_cached_memory reports the idle bytes held; gcg_release_cached_memory
 * returns them all to the driver (released_bytes, which may be NULL, receives
 * their count) and also trims the memory that the devices' default stream-ordered
 * pools keep for the library's temporaries (the sharder's sort buffers). */
int gcg_cached_memory(uint64_t *idle_device_bytes, uint64_t *idle_host_bytes);
int gcg_release_cached_memory(uint64_t *released_bytes);

/* Makes all later work on g run on `stream` (a cudaStream_t; NULL = legacy default). */
int gcg_graph_set_stream(gcg_graph *g, void *stream);

typedef struct {
    uint32_t num_vertices; /* graphchi_engine::num_vertices() (graphchi_engine.hpp:625-627) */
    uint32_t nshards;      /* intervals produced */
    uint64_t num_edges;    /* graphchi_engine::num_edges() */
    uint32_t has_out_csr;
    uint32_t reserved;
} gcg_graph_info;
int gcg_graph_get_info(const gcg_graph *g, gcg_graph_info *info);

/* Last vertex id of each interval: the contents of <base>.<P>.intervals
 * (sharder.hpp:909-920, read by load_vertex_intervals chifilenames.hpp:380-405).
 * last_vid: nshards entries, host or device. */
int gcg_graph_intervals(const gcg_graph *g, uint32_t *last_vid);

/* In/out degrees as struct degree {int indegree; int outdegree;} per vertex:
 * the contents of <base>_degs.bin (src/engine/auxdata/degree_data.hpp:45-48,
 * sharder.hpp:996-1006). pairs: 2*num_vertices int32, host or device. */
int gcg_graph_degrees(const gcg_graph *g, int32_t *pairs);

#define GCG_CSR_IN 0
#define GCG_CSR_OUT 1
/* Copies a CSR: rowptr (num_vertices+1) and col (num_edges), host or device. */
int gcg_graph_csr(const gcg_graph *g, int which, uint32_t *rowptr, uint32_t *col);

/* Dynamic graphs: replaces graphchi_dynamicgraph_engine's add_edge and edge
 * deletion (src/engine/dynamic_graphs/graphchi_dynamicgraph_engine.hpp:289-606:
 * added edges are buffered and merged into the shards, deleted edges are flagged
 * and dropped when a shard is rewritten). Here a batch of updates rebuilds the
 * resident graph on the device: afterwards it is exactly what gcg_graph_from_edges
 * would build, with the graph's own build flags and interval count, from its
 * edges plus the added ones (add) or minus every copy of the listed ones
 * (delete; absent edges are ignored). For a graph built with
 * GCG_BUILD_SYMMETRISE each edge is added or removed in both directions. Added
 * ids may exceed the vertex count, which then grows to max id + 1; deletion keeps
 * it. Cached plans (PageRank, CC) are rebuilt on their next use; the handle and
 * its stream stay. src/dst: m entries, host or device. */
int gcg_graph_add_edges(gcg_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t m);
int gcg_graph_delete_edges(gcg_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t m);

/* Borrowed device pointers to a graph's resident arrays, for callers that run
 * their own kernels over it (the functional plug-in of graphchi_gpu does). Valid
 * until gcg_graph_free; read-only; out_rowptr/out_col are NULL when the graph was
 * built without its out-edge CSR. No counterpart in the reference (its shards are
 * files). */
typedef struct {
    const uint32_t *in_rowptr, *in_col;   /* in-edges by destination, sources ascending */
    const uint32_t *out_rowptr, *out_col; /* out-edges by source, destinations ascending */
    const uint32_t *indeg, *outdeg;
    uint32_t num_vertices, reserved;
    uint64_t num_edges;
    void *stream; /* the graph's stream (cudaStream_t) */
} gcg_graph_device_view;
int gcg_graph_get_device_view(const gcg_graph *g, gcg_graph_device_view *view);

/* Writes the sharder's metadata files for `base`: <base>.<P>.intervals,
 * <base>.numvertices and <base>_degs.bin (sharder.hpp:909-926, :996-1006), so the
 * reference's readers (load_vertex_intervals, degree_data) accept the graph. */
int gcg_graph_write_metadata(const gcg_graph *g, const char *base);

/* Writes a vertex-value array as <base>.<elem_size>B.vout, the file
 * vertex_data_store writes and get_top_vertices / foreach_vertices /
 * sum_vertices / analyze_labels read (src/engine/auxdata/vertex_data.hpp:52-211,
 * src/api/chifilenames.hpp:65-71). values: host or device. */
int gcg_write_vout(const char *base, const void *values, uint32_t num_vertices, uint32_t elem_size);

/* ---- PageRank ---------------------------------------------------------- */

#define GCG_PR_JACOBI 0   /* bulk-synchronous (functional engine, sync mode) */
#define GCG_PR_GS_EXACT 1 /* vertex-API in-memory program (pagerank.cpp:121-146): Gauss-Seidel
                             in id order, bit-exact; the values are pr * outdeg as the app stores them */
#define GCG_PR_GS_EDGE 3  /* vertex-API edge-value program (pagerank.cpp:73-113, the app's choice when
                             num_vertices * 4 >= membudget): Gauss-Seidel in id order with
                             pagerank / outdeg (float) on the out-edges, bit-exact; the values are
                             the pageranks; delta_log gets each sweep's sum of |pagerank - old| */
#define GCG_PR_DELTA 2    /* selective scheduling: Jacobi sweeps over a device frontier
                             (bitset_scheduler.hpp:38-104): sweep 0 updates every vertex; a vertex
                             whose rank moved by more than delta_threshold x its rank schedules its
                             out-neighbours for the next sweep; stops when nothing is scheduled, at
                             tol or at max_sweeps. Needs the out-edge CSR. */

typedef struct {
    int mode;               /* GCG_PR_JACOBI, GCG_PR_GS_EXACT, GCG_PR_DELTA or GCG_PR_GS_EDGE */
    int max_sweeps;         /* update sweeps after the initial one (niters - 1) */
    double teleport;        /* added term: 0.15 (pagerank.cpp:94) or 0.15/N (pagerank_functional.cpp:74) */
    double damping;         /* 0.85 */
    double tol;             /* stop after the sweep whose normalised L1 change <= tol; 0 = run max_sweeps */
    float init;             /* initial vertex value when init_rank is NULL (1.0) */
    uint32_t flags;         /* GCG_PR_TIME_SWEEPS: time each sweep kernel with CUDA events */
    const float *init_rank; /* optional initial vector (num_vertices, host or device): the warm start */
    double *residuals;      /* optional: per-sweep residual log (max_sweeps doubles, host or device) */
    uint32_t source;        /* personalisation: teleport (and the initial mass 1) only at this
                               vertex; GCG_NO_SOURCE = plain PageRank. JACOBI only. */
    uint32_t reserved2;
    /* optional per-sweep progress log, the reference's write_delta_log line
     * "iteration,nupdates,work,delta" (graphchi_engine.hpp:593-599): delta_log[i] = sum over
     * vertices of |r' - r| in sweep i (FP64; graphchi_context::log_change, graphchi_context.hpp:82-106);
     * work_log[2i], [2i+1] = vertex updates and in-edges gathered up to and including sweep i
     * (GS_EDGE: in- plus out-edges, as the engine counts them for a program with edge values).
     * max_sweeps entries (2 x for work_log), host or device. JACOBI, DELTA and GS_EDGE modes. */
    double *delta_log;
    uint64_t *work_log;
    /* GCG_PR_DELTA: a vertex whose rank moved by more than delta_threshold x its new rank
     * schedules its out-neighbours for the next sweep */
    double delta_threshold;
} gcg_pr_params;

#define GCG_PR_TIME_SWEEPS 0x1u
/* Test hook of gcg_batch_pagerank: the persistent kernel's grid barrier waits for
 * one CTA that does not exist, so its bounded wait runs out and the call returns
 * GCG_ERR_TIMEOUT (exercises the failure path without faulting the GPU). */
#define GCG_PR_TEST_BARRIER_TIMEOUT 0x2u
#define GCG_NO_SOURCE 0xFFFFFFFFu

typedef struct {
    int sweeps;             /* sweeps run */
    int converged;          /* 1 if the tolerance was met */
    double residual;        /* normalised L1 change of the last sweep (double) */
    double device_ms;       /* device time of the sweeps (CUDA events on the graph's stream) */
    double sweep_kernel_ms; /* with GCG_PR_TIME_SWEEPS: summed time of the main sweep kernel */
    int timed_sweeps;       /* launches summed into sweep_kernel_ms */
    int kernel_launches;    /* kernels this call launched (early-exit launches included) */
    int levels;             /* GS modes: levels of the id-ordered dependency schedule (else 0) */
} gcg_pr_stats;

/* Fills params with the vertex-API defaults: Jacobi, teleport 0.15, damping 0.85,
 * init 1.0, 3 sweeps (niters 4, pagerank.cpp:155), tol 0. */
void gcg_pr_params_default(gcg_pr_params *p);

/* Replaces graphchi_engine::run(PagerankProgram / PagerankProgramInmem / the
 * functional pagerank_kernel, niters) (graphchi_engine.hpp:718-992,
 * example_apps/pagerank.cpp:73-144, example_apps/pagerank_functional.cpp:48-83).
 * JACOBI: r <- init; each sweep r[v] = (float)(teleport + damping * sum_{u->v}
 * r[u]/outdeg[u]) with float contributions and float sums, FP64 residual.
 * GS_EXACT: the in-memory vertex program's id-ordered Gauss-Seidel, writing the
 * same final values as pagerank.cpp:140-143 (pr * outdeg).
 * out_rank: num_vertices floats, host or device. stats may be NULL. */
int gcg_pagerank(gcg_graph *g, const gcg_pr_params *params, float *out_rank, gcg_pr_stats *stats);

/* Launch configuration of the Jacobi edge kernel of one graph (results do not
 * depend on it): hub_entries = shared-memory contribution cache entries (sources
 * whose out-degree rank is below it are read from shared memory; capped at the
 * plan's 49152), chunk_run = consecutive 256-edge chunks a warp takes at a time
 * (1 = warps stride chunk by chunk). Default: 41724 entries (the largest hub
 * that leaves the SM its 164 KB shared-memory carve-out, so L1 keeps ~92 KB) and
 * chunk_run 1, the fastest measured at R-MAT scale 24. gcg_pagerank_autotune
 * times `sweeps` fixed sweeps (the whole sweep, device time) of each candidate
 * (hub entries {0, 16384, 32768, 41724, 49152, the plan's} x runs {1, 2, 4, 16},
 * then 2..4 source tiers of the chosen hub, gcg_pagerank_set_tiers), keeps the
 * fastest for later calls on this graph and reports it (outputs may be NULL;
 * gcg_pagerank_get_tiers gives the tier count chosen). */
int gcg_pagerank_set_config(gcg_graph *g, uint32_t hub_entries, uint32_t chunk_run);
int gcg_pagerank_get_config(gcg_graph *g, uint32_t *hub_entries, uint32_t *chunk_run);
int gcg_pagerank_autotune(gcg_graph *g, int sweeps, uint32_t *hub_entries, uint32_t *chunk_run, double *ms_per_sweep);

/* Source tiers of the Jacobi edge phase (no counterpart in the reference; the
 * answers agree within float rounding: a row's sum is formed per tier, then the
 * tiers' partial sums are added in tier order). With `tiers` = t > 1 the
 * sources, relabelled by out-degree, are cut into tiers of hub_entries ids;
 * tier k >= 1 (ids [k h, (k+1) h)) gets its own edge array and edge pass with
 * its contributions in shared memory, tier 0 keeps the hub and every source past
 * the last tier. It trades one edge pass per tier for fewer scattered global
 * gathers. 1..4; 1 = one pass (the default). The tier arrays are built on the
 * first solve that uses them (one more copy of the column array). */
int gcg_pagerank_set_tiers(gcg_graph *g, uint32_t tiers);
int gcg_pagerank_get_tiers(gcg_graph *g, uint32_t *tiers);

/* Batched personalised PageRank (the engine's addition beside the reference's
 * one-vector runs of example_apps/pagerank.cpp): nsources sources solved together
 * as a vertex-major rank matrix. For source s: r_s starts at the indicator of
 * sources[s]; each sweep r_s[v] = (float)(params->teleport*[v == sources[s]] +
 * params->damping * sum_{u->v} r_s[u]/outdeg[u]) (float contributions and sums).
 * Each source stops on its own, as gcg_pagerank with params->source would: after
 * its first sweep whose normalised L1 change (FP64) is <= params->tol, or after
 * max_sweeps. Finished sources leave the matrix (it is compacted to the next
 * narrower width when the rest fit), so late sweeps gather shorter rows.
 * mode must be GCG_PR_JACOBI, init_rank NULL and source GCG_NO_SOURCE.
 * sources: nsources ids, host or device. out: num_vertices x nsources floats,
 * out[v * nsources + s], host or device. params->residuals (if set) receives the
 * per-sweep maximum residual of the sources still iterating; params->work_log
 * (if set, 2 x max_sweeps entries) the cumulative work: work_log[2i] = vertex
 * updates and work_log[2i+1] = in-edges gathered, summed over the sources still
 * iterating in sweeps 0..i (V and E per source and sweep). stats->sweeps is
 * the largest per-source count. Sources run in groups of 256. */
int gcg_ppr_batched(gcg_graph *g, const uint32_t *sources, uint32_t nsources, const gcg_pr_params *params,
                    float *out, gcg_pr_stats *stats);

/* ---- many graphs in one persistent launch -------------------------------- */

/* A batch of independent graphs (the engine's addition: the reference runs one
 * graph per engine, graphchi_engine.hpp:148). gcg_batch_create concatenates the
 * graphs' in-edge CSRs into one block-diagonal union on the device (each graph
 * is one interval of it); the graphs may be freed afterwards. Up to 1024 graphs,
 * 2^32-1 vertices and edges in total. */
typedef struct gcg_batch gcg_batch;
int gcg_batch_create(gcg_graph *const *graphs, uint32_t ngraphs, gcg_batch **out);
/* The same with flags. GCG_BATCH_ONE_HUB: relabel the union's sources by
 * out-degree over the whole union (one shared-memory hub holding the union's
 * hottest sources, rows kept in id order) instead of within each graph's id
 * range (a hub per graph, rows in relabelled order; the default, and the only
 * layout whose ranks are bit-identical to each graph's own gcg_pagerank solve).
 * Without the flag the one-hub layout is taken only when the union's ids are too
 * wide for per-graph relabelling (more than 64 sort-key bits). */
#define GCG_BATCH_ONE_HUB 1u
int gcg_batch_create_ex(gcg_graph *const *graphs, uint32_t ngraphs, uint32_t flags, gcg_batch **out);
/* First union vertex id of each graph (ngraphs+1 entries, last = total). */
int gcg_batch_vertex_offsets(const gcg_batch *b, uint64_t *offsets);
int gcg_batch_set_stream(gcg_batch *b, void *stream);
/* Jacobi PageRank of every graph (the gcg_pagerank formula and stopping rule per
 * graph, bit-identical results) in ONE cooperative persistent kernel: sweeps
 * proceed together, a graph leaves the device work queues when its own residual
 * is <= tol. out_ranks: total vertices, graph g at its vertex offset (may be
 * NULL); sweeps / residuals: per graph (may be NULL); params->init_rank (total
 * vertices) may seed all graphs. Without init_rank the whole solve is captured
 * into a CUDA graph on the first call with a given parameter set and replayed on
 * later calls. Returns GCG_ERR_TIMEOUT if a bounded grid-barrier wait runs out.
 * Until gcg_batch_set_stream is called, the batch runs on a stream of its own
 * that waits for the legacy default stream at the start of every call. */
int gcg_batch_pagerank(gcg_batch *b, const gcg_pr_params *params, float *out_ranks, int32_t *sweeps,
                       double *residuals, gcg_pr_stats *stats);
/* Autotuner of the persistent launch: times `sweeps` fixed sweeps of each
 * candidate configuration and keeps the fastest for later solves (results do not
 * depend on it). Candidates: shared-memory hub entries per graph (each graph's
 * sources whose out-degree rank within the graph is below it are read from
 * shared memory: the degree threshold of the cache) in {0, 8192, 16384, 32768,
 * 41724, 49152, the plan's}. CTAs take ranges of the active graphs' chunks from a
 * device cursor, large ranges first and smaller ones as the work runs out. Only when the union's ids are too wide for per-graph relabelling
 * (more than 64 sort-key bits) is there one hub over the union's hottest sources
 * and the edge phase's work distribution a second candidate: warps striding over
 * the chunks (queue_run 0) or taking runs of 1, 4 or 16 chunks from a device
 * work queue. Outputs may be NULL. */
int gcg_batch_autotune(gcg_batch *b, int sweeps, uint32_t *hub_entries, uint32_t *queue_run, double *ms_per_sweep);
/* Sets the configuration by hand (hub entries are capped at the plan's;
 * queue_run applies to the one-hub layout only). */
int gcg_batch_set_config(gcg_batch *b, uint32_t hub_entries, uint32_t queue_run);
/* The configuration in use, and whether a captured solve is ready to replay. */
int gcg_batch_get_config(const gcg_batch *b, uint32_t *hub_entries, uint32_t *queue_run, int *graph_ready);
int gcg_batch_free(gcg_batch *b);

/* No counterpart in the reference. PageRank (GCG_PR_JACOBI only) over an in-edge
 * CSR the caller already keeps in device memory, for callers that cannot let a
 * library allocate device memory (a host framework whose own allocator owns the
 * GPU, or a loop that must not incur cudaMalloc/cudaFree synchronisation). It
 * allocates nothing: in_rowptr (num_vertices+1), in_col, outdeg (num_vertices),
 * out_rank (num_vertices) and the optional params->init_rank / residuals must all
 * be device memory of the current device (or managed memory), or the call fails
 * with GCG_ERR_INVALID. Its scratch is a fixed static device
 * array sized for GCG_NOALLOC_MAX_VERTICES vertices (about 12.6 MB, held by every
 * GPU that loads the library); larger graphs are rejected with
 * GCG_ERR_UNSUPPORTED. The first call on a device looks up that array's address;
 * make it before any stream capture. All calls share the array: calls that
 * overlap on the GPU race. Each call waits for `stream` before it returns.
 * residuals[i] is written for the sweeps that ran (i < stats->sweeps) only;
 * stats->device_ms is read from the GPU's global timer (start of the first
 * kernel to the end of the last sweep). stream: a cudaStream_t (NULL = legacy
 * default). */
#define GCG_NOALLOC_MAX_VERTICES (1u << 20)
int gcg_pagerank_csr_noalloc(const uint32_t *in_rowptr, const uint32_t *in_col, const uint32_t *outdeg,
                             uint32_t num_vertices, const gcg_pr_params *params, float *out_rank,
                             void *stream, gcg_pr_stats *stats);

/* ---- learned warm start ------------------------------------------------- */

/* No counterpart in the reference (its PageRank starts from a constant,
 * example_apps/pagerank.cpp:80-85). A small MLP maps 8 per-vertex degree
 * features to log(rank / teleport); exp of its output, times teleport, seeds the
 * Jacobi iteration through gcg_pr_params.init_rank. The iteration then runs to
 * the same residual as from the uniform start, so the answer keeps its accuracy.
 *
 * Features of vertex v (raw, before the model's normalisation), with
 * L(u) = log(1 + indeg(u)):
 *   0 log(1 + indeg v)        1 log(1 + outdeg v)
 *   2 mean of L(u) over in-neighbours u (0 without in-edges)
 *   3 max of L(u) over in-neighbours u (0 without in-edges)
 *   4 log(1 + sum of indeg(u) over in-neighbours u)   (2-hop in-degree)
 *   5 1 / outdeg v (0 without out-edges)
 *   6, 7 bits B-1 and B-2 of v, B = bits of a vertex id (R-MAT quadrant bits)
 *
 * Network: x' = bf16((x - mean) * inv_std); h1 = bf16(relu(W1 x' + b1));
 * h2 = relu(W2 h1 + b2); y = W3 . h2 + b3, with W1 (64x8), W2 (64x64), W3 (64)
 * rounded to BF16 and every product summed in FP32. Parameters, flat FP32 in this
 * order: W1 [64][8] (row = hidden unit), b1 [64], W2 [64][64] (row = output
 * unit), b2 [64], W3 [64], b3 [1]. Training keeps FP32 master weights and runs
 * Adam on the loss mean((y - target)^2), gradients passed straight through the
 * BF16 roundings. */
#define GCG_MLP_IN 8
#define GCG_MLP_HIDDEN 64
#define GCG_MLP_NPARAMS (64 * 8 + 64 + 64 * 64 + 64 + 64 + 1)
typedef struct gcg_mlp gcg_mlp;

typedef struct {
    uint32_t epochs;     /* passes over the samples */
    uint32_t batch;      /* samples per Adam step (multiple of 128) */
    float lr, beta1, beta2, eps;
    uint64_t seed;       /* sample order */
} gcg_mlp_train_params;

/* He-initialised weights (seeded), zero biases, identity normalisation. */
int gcg_mlp_create(uint64_t seed, gcg_mlp **out);
int gcg_mlp_free(gcg_mlp *m);
/* params: GCG_MLP_NPARAMS floats; norm: 16 floats (mean[8], inv_std[8]); either may be NULL. */
int gcg_mlp_get(const gcg_mlp *m, float *params, float *norm);
int gcg_mlp_set(gcg_mlp *m, const float *params, const float *norm);
/* Sets the normalisation from n samples (x: n x 8, row-major, host or device). */
int gcg_mlp_fit_normalisation(gcg_mlp *m, const float *x, uint64_t n);
/* Raw features of every vertex: features[v * 8 + i], host or device. */
int gcg_warm_features(gcg_graph *g, float *features);
/* Network output y for n samples (training kernel's forward, FP32 CUDA cores). */
int gcg_mlp_forward(const gcg_mlp *m, const float *x, uint64_t n, float *y);
/* Gradient of mean((y - t)^2) over n samples w.r.t. the parameters (the training
 * kernels, without an update): grad GCG_MLP_NPARAMS floats; *loss the mean loss. */
int gcg_mlp_gradient(const gcg_mlp *m, const float *x, const float *t, uint64_t n, float *grad, double *loss);
/* Minibatch Adam over n samples; epoch_loss (epochs floats, may be NULL) receives
 * the mean training loss of each epoch. */
void gcg_mlp_train_params_default(gcg_mlp_train_params *p);
int gcg_mlp_train(gcg_mlp *m, const float *x, const float *t, uint64_t n, const gcg_mlp_train_params *p,
                  float *epoch_loss);
/* The warm start: features and network fused on the device (tensor-core
 * inference), p_v = teleport * exp(y_v) for a vertex with in-edges and exactly
 * teleport for one without (its rank after any sweep). The predictions p are then
 * scaled by one factor alpha chosen so that a Jacobi sweep keeps the total rank
 * (with Z = vertices without in-edges, D = without out-edges, M = sum of p
 * outside Z, M_D = its part on D: alpha = teleport*(n - (1-damping)|Z| -
 * damping|Z&D|) / ((1-damping)M + damping M_D)); a per-graph bias of the network
 * would otherwise excite the slowest mode of the iteration. init_rank:
 * num_vertices, host or device. *device_ms (may be NULL) receives the device time. */
int gcg_warm_start_rank(gcg_graph *g, const gcg_mlp *m, double teleport, double damping, float *init_rank,
                        double *device_ms);

/* ---- connected components ---------------------------------------------- */

typedef struct {
    int passes;        /* edge passes run */
    uint32_t ncomponents;
    double device_ms;
} gcg_cc_stats;

/* Replaces graphchi_engine::run(ConnectedComponentsProgram, niters)
 * (example_apps/connectedcomponents.cpp:79-138): labels = the fixpoint of
 * min-label propagation over in- and out-edges, i.e. the minimum vertex id of
 * each weakly connected component. labels: num_vertices, host or device. */
int gcg_connected_components(gcg_graph *g, uint32_t *labels, gcg_cc_stats *stats);

#define GCG_CC_UNION_FIND 0        /* hook-and-compress (gcg_connected_components) */
#define GCG_CC_LABEL_PROPAGATION 1 /* the reference's update rule, iterated to its fixpoint */
typedef struct {
    int algorithm;      /* GCG_CC_UNION_FIND or GCG_CC_LABEL_PROPAGATION */
    int scheduler;      /* label propagation: 1 = selective scheduling on a device frontier, as the
                           reference's scheduler=1 (bitset_scheduler.hpp:38-104): only vertices whose
                           label may drop are updated; 0 = every vertex every iteration */
    int max_iterations; /* label propagation: cap (0 = 1000, connectedcomponents.cpp:165) */
    uint32_t reserved;
    int32_t *frontier_log; /* optional: per iteration, vertices updated (max_iterations ints, host or device) */
} gcg_cc_params;
/* Same labels as gcg_connected_components (the minimum id per weak component)
 * by the chosen algorithm; label propagation needs whole neighbourhoods (a graph
 * built with GCG_BUILD_SYMMETRISE, or with its out-edge CSR). stats->passes =
 * iterations run. */
int gcg_connected_components_ex(gcg_graph *g, const gcg_cc_params *p, uint32_t *labels, gcg_cc_stats *stats);

/* ---- triangle counting ------------------------------------------------- */

typedef struct {
    uint64_t triangles;
    uint64_t oriented_edges; /* undirected simple edges after orientation */
    double device_ms;
} gcg_tc_stats;

/* Replaces order_by_degree + graphchi_dynamicgraph_engine::run(
 * TriangleCountingProgram) + sum_vertices/3
 * (src/preprocessing/util/orderbydegree.hpp:59-143,
 * example_apps/trianglecounting.cpp:288-477). Vertices are ranked by
 * (in+out degree, id); vertexmap[v] = rank (<base>.vertexmap); per_rank[r] = the
 * number of triangles through the vertex of rank r (<base>_degord.4B.vout).
 * total, per_rank and vertexmap may each be NULL; arrays host or device. */
int gcg_triangle_count(gcg_graph *g, uint64_t *total, uint32_t *per_rank, uint32_t *vertexmap,
                       gcg_tc_stats *stats);

/* ---- synthetic inputs -------------------------------------------------- */

/* R-MAT edges (quadrant probabilities a, b, c, d = 1-a-b-c), m edges over
 * 2^scale vertices, seeded; src/dst: m entries each, host or device (device
 * arrays are filled by a kernel, host arrays by host threads: identical). */
int gcg_generate_rmat(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed,
                      uint32_t *src, uint32_t *dst);

/* Erdos-Renyi G(n, m) edges (uniform src and dst in [0, n)), seeded. */
int gcg_generate_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *src, uint32_t *dst);

/* ---- errors ------------------------------------------------------------ */

/* Message of the last failure on this thread ("" if none). Replaces the
 * reference's logstream(LOG_FATAL)/assert exits with a returned status. */
const char *gcg_last_error(void);

/* Library version string. */
const char *gcg_version(void);

#ifdef __cplusplus
}
#endif
#endif
