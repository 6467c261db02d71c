/*
 * ORACLE — test infrastructure only. A plain-C, single-threaded restatement of
 * the GraphChi parallel-sliding-windows hot path (sharder -> engine -> update()
 * of PageRank, connected components and triangle counting). Only tests/, the
 * smoke check and bench.py's CPU-baseline leg may load it, and only as the
 * checker; the product path never calls it.
 *
 * Pinned against the compiled reference (oracle/_ref) through the golden
 * fixtures in tests/golden/ (see tests/test_oracle_golden.py).
 * Every function cites the reference file:line it restates.
 */
#ifndef GCG_ORACLE_H
#define GCG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Writes a "src\tdst" edge list (input of convert_edgelist). 0 on success. */
int orc_write_edgelist(const char *path, const uint32_t *src, const uint32_t *dst, uint64_t m);

/* Canonical edge set as the sharder sees it: drops self-loops
 * (src/preprocessing/sharder.hpp:428-431); with symmetrise adds (v,u) for every
 * (u,v); with dedup sorts by (src,dst) and keeps one copy. Without dedup the
 * input order is kept (mirrored edges appended after the originals).
 * out_* must hold 2*m entries when symmetrise, m otherwise. Returns the count. */
uint64_t orc_canonical_edges(const uint32_t *src, const uint32_t *dst, uint64_t m,
                             int symmetrise, int dedup, uint32_t *out_src, uint32_t *out_dst);

/* CSR grouped by dst (by_dst=1: in-edges, col = src) or by src (by_dst=0:
 * out-edges, col = dst); each row's column list ascending (multi-edges kept).
 * rowptr has nv+1 entries. */
void orc_build_csr(uint32_t nv, const uint32_t *src, const uint32_t *dst, uint64_t m,
                   int by_dst, uint32_t *rowptr, uint32_t *col);

/* Interval split of the sharder's k-way merge sink
 * (src/preprocessing/sharder.hpp:861-892, initial edges_per_shard :962, last
 * interval end :880): returns the number of intervals and writes the last vertex
 * id of each into last_vid (nshards entries). max_vid = numvertices-1. */
uint32_t orc_intervals(const uint32_t *in_rowptr, uint32_t nv, uint32_t nshards, uint32_t *last_vid);

/* Number of shards chosen by nshards="auto"
 * (src/preprocessing/sharder.hpp:563-575) for edge-value size esize. */
uint32_t orc_auto_nshards(uint64_t nedges, uint32_t esize, uint32_t membudget_mb);

/* Vertex-API PageRank, in-memory program (example_apps/pagerank.cpp:121-146)
 * under the engine's deterministic id-ordered execution
 * (src/engine/graphchi_engine.hpp:396-454): sequential Gauss-Seidel in vertex id
 * order, in-edges summed in ascending source order in float, apply in double
 * rounded to float. Writes the final vertex values (pr*outc on the last
 * iteration, pagerank.cpp:140-143). niters counts iteration 0 (the init). */
void orc_pagerank_gs_inmem(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                           const uint32_t *outdeg, int niters, float *out_values);

/* Vertex-API PageRank, edge-value program (example_apps/pagerank.cpp:73-113,
 * chosen by the app when num_vertices * 4 >= membudget, :166-177) under the
 * engine's id-ordered execution: sequential Gauss-Seidel where every out-edge of
 * u holds u's pagerank / outdeg (float division), initially (float)(1.0/outdeg);
 * the vertex value is pagerank = (float)(0.15 + 0.85*(double)sum). out_values:
 * vertex values after niters iterations (iteration 0 = the initialisation);
 * delta_log (may be NULL, niters entries): each iteration's sum of
 * |pagerank - old| (float differences added in double in vertex order), the
 * value graphchi_engine writes to <base>.deltalog. */
void orc_pagerank_gs_edge(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                          const uint32_t *outdeg, int niters, float *out_values, double *delta_log);

/* Either vertex-API program (edge 0: in-memory, edge 1: edge values) with
 * per-sweep tracking of the pageranks (float)(0.15 + 0.85*(double)sum):
 * delta_log[k] = sum |pagerank - previous|, res_log[k] = that / sum |pagerank|
 * (either may be NULL); stops after the first sweep with residual <= tol (tol >
 * 0) or after max_sweeps sweeps (iterations after the initial one). out_values
 * as the app stores them. Returns the sweeps run. */
int orc_pagerank_gs_track(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                          const uint32_t *outdeg, int edge, int max_sweeps, double tol,
                          float *out_values, double *delta_log, double *res_log);

/* Bulk-synchronous PageRank with the functional kernel contract
 * (src/api/functional/functional_bulksync.hpp:91-113,
 * example_apps/pagerank_functional.cpp:51-81): init value `init`; each sweep
 * gathers old value/outdeg of in-neighbours (float sum, ascending source), applies
 * (float)(teleport + damping*(double)sum), scatters v/outdeg in float.
 * Runs up to max_sweeps sweeps; with tol > 0 stops after the first sweep whose
 * normalised L1 change sum|new-old|/sum|new| (double) is <= tol. res_log (may be
 * NULL) receives each sweep's residual. Returns the number of sweeps run. */
int orc_pagerank_jacobi(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                        const uint32_t *outdeg, double teleport, double damping, float init,
                        int max_sweeps, double tol, float *out_rank, double *res_log);

/* Same iteration entirely in double (the FP64 reference used to state error). */
int orc_pagerank_jacobi_f64(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                            const uint32_t *outdeg, double teleport, double damping, double init,
                            int max_sweeps, double tol, double *out_rank);

/* Connected components by min-label propagation
 * (example_apps/connectedcomponents.cpp:79-138): labels start at the vertex id,
 * every sweep visits vertices in id order (Gauss-Seidel, the engine's
 * deterministic order) and takes the minimum over all in- and out-neighbours,
 * until a sweep changes nothing. Returns the number of sweeps. */
int orc_cc(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
           const uint32_t *out_rowptr, const uint32_t *out_col, uint32_t *labels);

/* Triangle counting as example_apps/trianglecounting.cpp computes it:
 * vertices ranked by (in+out degree, id) ascending
 * (src/preprocessing/util/orderbydegree.hpp:16-25,71-89), vertexmap[v] = rank;
 * every triangle adds one to each of its three corners' counts in rank space
 * (the per-vertex values of <file>_degord.4B.vout, trianglecounting.cpp:288-357).
 * per_rank (nv entries) and vertexmap (nv entries) may be NULL.
 * Returns the number of triangles (sum of counts / 3, trianglecounting.cpp:476-477). */
uint64_t orc_tc(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                const uint32_t *out_rowptr, const uint32_t *out_col,
                uint32_t *per_rank, uint32_t *vertexmap);

/* Personalised PageRank for k sources (no reference counterpart; the semantics
 * of the batched GPU path): r_s starts at e_s; each sweep
 * r_s[v] = (float)((1-damping)*[v==s] + damping*(double)sum_{u->v} c_s[u]) with
 * c_s[u] = r_s[u]/outdeg[u] in float and the float sum in ascending source order.
 * Each source stops (its column is frozen) after its own first sweep where
 * sum|new-old|/sum|new| <= tol; all stop after max_sweeps. out is vertex-major
 * (out[v*k + s]). Returns the number of sweeps of the slowest source. */
int orc_ppr(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
            const uint32_t *outdeg, const uint32_t *sources, uint32_t k, double damping,
            int max_sweeps, double tol, float *out);

/* ---- multithreaded variants (OpenMP) for checks at full size ---- */

/* The library's seeded R-MAT generator (csrc/gcg_rng.h) restated: m raw edges
 * (self-loops and duplicates included), bit-identical to the library's. */
void orc_rmat_edges(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed,
                    uint32_t *src, uint32_t *dst);

/* orc_pagerank_jacobi with rows split across threads: bit-identical ranks; the
 * residual's FP64 sums are formed in fixed 65536-row blocks added in order. */
int orc_pagerank_jacobi_mt(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                           const uint32_t *outdeg, double teleport, double damping, float init,
                           int max_sweeps, double tol, float *out_rank, double *res_log);

/* orc_pagerank_jacobi_f64 with rows split across threads; init_vec (NULL: the
 * constant init) is the starting vector; res_log (may be NULL) the residuals. */
int orc_pagerank_jacobi_f64_mt(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                               const uint32_t *outdeg, double teleport, double damping, double init,
                               const double *init_vec, int max_sweeps, double tol, double *out_rank,
                               double *res_log);

/* The in-CSR (and out-degrees) of the canonical edge set -- the arrays of
 * orc_canonical_edges(dedup) + orc_build_csr(by_dst=1) -- built with a
 * multithreaded radix sort. Ids must be < nv_cap; rowptr holds nv_cap+1
 * entries, col m, outdeg nv_cap. Writes nv (max id + 1); returns E. */
uint64_t orc_in_csr_mt(const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t nv_cap,
                       uint32_t *nv_out, uint32_t *rowptr, uint32_t *col, uint32_t *outdeg);

#ifdef __cplusplus
}
#endif
#endif
