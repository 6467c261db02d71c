/*
 * ORACLE — test infrastructure only (see oracle.h). Plain C restatement of the
 * GraphChi PSW hot path; each function cites the reference file:line it follows.
 * Single-threaded and written for clarity, not speed, except the _mt variants at
 * the end (OpenMP over rows or edges, same results) used for full-size checks.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- helpers ------------------------------------------------------------ */

/* LSD radix sort of 64-bit keys, 16-bit digits (4 passes), stable. */
static void radix_sort_u64(uint64_t *a, uint64_t n) {
    if (n < 2) return;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *cnt = (uint64_t *)malloc(65536 * sizeof(uint64_t));
    uint64_t *src = a, *dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        int sh = 16 * pass;
        memset(cnt, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xFFFF]++;
        uint64_t run = 0;
        for (int d = 0; d < 65536; ++d) { uint64_t c = cnt[d]; cnt[d] = run; run += c; }
        for (uint64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        uint64_t *t = src; src = dst; dst = t;
    }
    /* 4 passes: result is back in a */
    free(tmp);
    free(cnt);
}

static int cmp_u32(const void *x, const void *y) {
    uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
    return (a > b) - (a < b);
}

/* Writes "src\tdst\n" lines (the edge-list input of convert_edgelist). */
int orc_write_edgelist(const char *path, const uint32_t *src, const uint32_t *dst, uint64_t m) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    char buf[1 << 16];
    size_t pos = 0;
    for (uint64_t i = 0; i < m; ++i) {
        char tmp[32];
        int n = 0;
        uint32_t a = src[i], b = dst[i];
        char t1[12], t2[12];
        int l1 = 0, l2 = 0;
        do { t1[l1++] = (char)('0' + a % 10); a /= 10; } while (a);
        do { t2[l2++] = (char)('0' + b % 10); b /= 10; } while (b);
        while (l1) tmp[n++] = t1[--l1];
        tmp[n++] = '\t';
        while (l2) tmp[n++] = t2[--l2];
        tmp[n++] = '\n';
        if (pos + (size_t)n > sizeof(buf)) { fwrite(buf, 1, pos, f); pos = 0; }
        memcpy(buf + pos, tmp, (size_t)n);
        pos += (size_t)n;
    }
    fwrite(buf, 1, pos, f);
    return fclose(f) == 0 ? 0 : -1;
}

/* ---- sharder ------------------------------------------------------------ */

uint64_t orc_canonical_edges(const uint32_t *src, const uint32_t *dst, uint64_t m,
                             int symmetrise, int dedup, uint32_t *out_src, uint32_t *out_dst) {
    uint64_t n = 0;
    for (uint64_t i = 0; i < m; ++i) {
        if (src[i] == dst[i]) continue; /* sharder.hpp:428-431 */
        out_src[n] = src[i];
        out_dst[n] = dst[i];
        ++n;
    }
    if (symmetrise) {
        uint64_t n0 = n;
        for (uint64_t i = 0; i < n0; ++i) {
            out_src[n] = out_dst[i];
            out_dst[n] = out_src[i];
            ++n;
        }
    }
    if (dedup && n > 0) {
        uint64_t *k = (uint64_t *)malloc(n * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; ++i) k[i] = ((uint64_t)out_src[i] << 32) | out_dst[i];
        radix_sort_u64(k, n);
        uint64_t w = 0;
        for (uint64_t i = 0; i < n; ++i) {
            if (i > 0 && k[i] == k[i - 1]) continue;
            out_src[w] = (uint32_t)(k[i] >> 32);
            out_dst[w] = (uint32_t)k[i];
            ++w;
        }
        free(k);
        n = w;
    }
    return n;
}

void orc_build_csr(uint32_t nv, const uint32_t *src, const uint32_t *dst, uint64_t m,
                   int by_dst, uint32_t *rowptr, uint32_t *col) {
    const uint32_t *row = by_dst ? dst : src;
    const uint32_t *oth = by_dst ? src : dst;
    memset(rowptr, 0, (size_t)(nv + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < m; ++i) rowptr[row[i] + 1]++;
    for (uint32_t v = 0; v < nv; ++v) rowptr[v + 1] += rowptr[v];
    uint32_t *fill = (uint32_t *)malloc((size_t)(nv + 1) * sizeof(uint32_t));
    memcpy(fill, rowptr, (size_t)(nv + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < m; ++i) col[fill[row[i]]++] = oth[i];
    free(fill);
    for (uint32_t v = 0; v < nv; ++v) {
        uint32_t b = rowptr[v], e = rowptr[v + 1];
        int sorted = 1;
        for (uint32_t j = b + 1; j < e && sorted; ++j) sorted = col[j - 1] <= col[j];
        if (!sorted) qsort(col + b, e - b, sizeof(uint32_t), cmp_u32);
    }
}

uint32_t orc_intervals(const uint32_t *in_rowptr, uint32_t nv, uint32_t nshards, uint32_t *last_vid) {
    uint64_t E = in_rowptr[nv];
    uint32_t max_vid = nv - 1;
    if (E == 0 || nshards <= 1) {
        last_vid[0] = max_vid;
        return 1;
    }
    /* sharder.hpp:962: edges_per_shard = shoveled_edges / nshards + 1 */
    uint64_t edges_per_shard = E / nshards + 1;
    uint64_t cur = 0, sharded = 0;
    uint32_t shardnum = 0;
    uint32_t prevvid = 0xFFFFFFFFu;
    for (uint32_t v = 0; v < nv; ++v) {
        uint64_t d = (uint64_t)in_rowptr[v + 1] - in_rowptr[v];
        if (d == 0) continue;
        /* sharder.hpp:862: cut before the first edge of a new dst once full */
        if (cur >= edges_per_shard && v != prevvid) {
            last_vid[shardnum] = (shardnum == nshards - 1) ? max_vid : prevvid; /* :880 */
            ++shardnum;
            cur = 0;
            if (shardnum < nshards) edges_per_shard = (E - sharded) / (nshards - shardnum); /* :889 */
        }
        cur += d;
        sharded += d;
        prevvid = v;
    }
    /* done() -> createnextshard() (sharder.hpp:894-895) */
    last_vid[shardnum] = (shardnum == nshards - 1) ? max_vid : prevvid;
    ++shardnum;
    return shardnum;
}

uint32_t orc_auto_nshards(uint64_t nedges, uint32_t esize, uint32_t membudget_mb) {
    double max_shardsize = membudget_mb * 1024. * 1024. / 8;
    return (uint32_t)(1 + ((double)(nedges * esize) / max_shardsize) + 0.5);
}

/* ---- PageRank ----------------------------------------------------------- */

void orc_pagerank_gs_inmem(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                           const uint32_t *outdeg, int niters, float *out_values) {
    const double RESET = 0.15; /* pagerank.cpp:43 RANDOMRESETPROB */
    float *pr = (float *)malloc((size_t)nv * sizeof(float));
    for (uint32_t v = 0; v < nv; ++v) pr[v] = (float)RESET; /* pagerank.cpp:124 */
    for (int it = 0; it < niters; ++it) {
        for (uint32_t v = 0; v < nv; ++v) {
            int outc = (int)outdeg[v];
            if (it > 0) { /* pagerank.cpp:127-136 */
                float sum = 0.0f;
                for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += pr[in_col[j]];
                if (outc > 0)
                    pr[v] = (float)((RESET + (1 - RESET) * (double)sum) / (double)outc);
                else
                    pr[v] = (float)(RESET + (1 - RESET) * (double)sum);
            } else { /* pagerank.cpp:137-139 */
                if (outc > 0) pr[v] = 1.0f / (float)outc;
            }
            if (it == niters - 1) /* pagerank.cpp:140-143 */
                out_values[v] = outc > 0 ? pr[v] * (float)outc : pr[v];
        }
    }
    free(pr);
}

int orc_pagerank_jacobi(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                        const uint32_t *outdeg, double teleport, double damping, float init,
                        int max_sweeps, double tol, float *out_rank, double *res_log) {
    float *r = (float *)malloc((size_t)nv * sizeof(float));
    float *c = (float *)malloc((size_t)nv * sizeof(float));
    float *cn = (float *)malloc((size_t)nv * sizeof(float));
    for (uint32_t v = 0; v < nv; ++v) { /* iteration 0: initial_value + scatter */
        r[v] = init;
        c[v] = outdeg[v] ? r[v] / (float)outdeg[v] : 0.0f;
    }
    int sweeps = 0;
    for (int s = 0; s < max_sweeps; ++s) {
        double dsum = 0, nsum = 0;
        for (uint32_t v = 0; v < nv; ++v) {
            float sum = 0.0f; /* functional_bulksync.hpp:91-101 gather (plus) */
            for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
            float nvv = (float)(teleport + damping * (double)sum); /* apply */
            dsum += fabs((double)nvv - (double)r[v]);
            nsum += fabs((double)nvv);
            r[v] = nvv;
            cn[v] = outdeg[v] ? nvv / (float)outdeg[v] : 0.0f; /* value_to_neighbor */
        }
        float *t = c; c = cn; cn = t;
        ++sweeps;
        double res = nsum > 0 ? dsum / nsum : 0.0;
        if (res_log) res_log[s] = res;
        if (tol > 0 && res <= tol) break;
    }
    memcpy(out_rank, r, (size_t)nv * sizeof(float));
    free(r); free(c); free(cn);
    return sweeps;
}

int orc_pagerank_jacobi_f64(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                            const uint32_t *outdeg, double teleport, double damping, double init,
                            int max_sweeps, double tol, double *out_rank) {
    double *r = (double *)malloc((size_t)nv * sizeof(double));
    double *c = (double *)malloc((size_t)nv * sizeof(double));
    double *cn = (double *)malloc((size_t)nv * sizeof(double));
    for (uint32_t v = 0; v < nv; ++v) {
        r[v] = init;
        c[v] = outdeg[v] ? r[v] / outdeg[v] : 0.0;
    }
    int sweeps = 0;
    for (int s = 0; s < max_sweeps; ++s) {
        double dsum = 0, nsum = 0;
        for (uint32_t v = 0; v < nv; ++v) {
            double sum = 0.0;
            for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
            double x = teleport + damping * sum;
            dsum += fabs(x - r[v]);
            nsum += fabs(x);
            r[v] = x;
            cn[v] = outdeg[v] ? x / outdeg[v] : 0.0;
        }
        double *t = c; c = cn; cn = t;
        ++sweeps;
        if (tol > 0 && nsum > 0 && dsum / nsum <= tol) break;
    }
    memcpy(out_rank, r, (size_t)nv * sizeof(double));
    free(r); free(c); free(cn);
    return sweeps;
}

/* ---- connected components ---------------------------------------------- */

int orc_cc(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
           const uint32_t *out_rowptr, const uint32_t *out_col, uint32_t *labels) {
    for (uint32_t v = 0; v < nv; ++v) labels[v] = v; /* connectedcomponents.cpp:83-86 */
    int sweeps = 0;
    int changed = 1;
    while (changed) {
        changed = 0;
        ++sweeps;
        for (uint32_t v = 0; v < nv; ++v) { /* :89-97 min over all incident edges */
            uint32_t m = labels[v];
            for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j)
                if (labels[in_col[j]] < m) m = labels[in_col[j]];
            for (uint32_t j = out_rowptr[v]; j < out_rowptr[v + 1]; ++j)
                if (labels[out_col[j]] < m) m = labels[out_col[j]];
            if (m < labels[v]) { labels[v] = m; changed = 1; } /* :107-115, :125-138 */
        }
    }
    return sweeps;
}

/* ---- triangle counting -------------------------------------------------- */

uint64_t orc_tc(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                const uint32_t *out_rowptr, const uint32_t *out_col,
                uint32_t *per_rank, uint32_t *vertexmap) {
    /* orderbydegree.hpp:71-89: deg = in + out; sort by (deg, id); rank = position */
    uint64_t *key = (uint64_t *)malloc((size_t)nv * sizeof(uint64_t));
    for (uint32_t v = 0; v < nv; ++v) {
        uint64_t deg = (uint64_t)(in_rowptr[v + 1] - in_rowptr[v]) + (out_rowptr[v + 1] - out_rowptr[v]);
        key[v] = (deg << 32) | v;
    }
    radix_sort_u64(key, nv);
    uint32_t *rank = (uint32_t *)malloc((size_t)nv * sizeof(uint32_t));
    for (uint32_t i = 0; i < nv; ++i) rank[(uint32_t)key[i]] = i;
    free(key);
    if (vertexmap) memcpy(vertexmap, rank, (size_t)nv * sizeof(uint32_t));

    /* undirected simple graph in rank space, oriented low -> high rank */
    uint64_t m = out_rowptr[nv];
    uint64_t *pairs = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    for (uint32_t u = 0; u < nv; ++u)
        for (uint32_t j = out_rowptr[u]; j < out_rowptr[u + 1]; ++j) {
            uint32_t a = rank[u], b = rank[out_col[j]];
            if (a > b) { uint32_t t = a; a = b; b = t; }
            pairs[j] = ((uint64_t)a << 32) | b;
        }
    radix_sort_u64(pairs, m);
    uint64_t w = 0;
    for (uint64_t i = 0; i < m; ++i) {
        if (i > 0 && pairs[i] == pairs[i - 1]) continue;
        if ((uint32_t)(pairs[i] >> 32) == (uint32_t)pairs[i]) continue;
        pairs[w++] = pairs[i];
    }
    uint32_t *rp = (uint32_t *)calloc((size_t)nv + 1, sizeof(uint32_t));
    uint32_t *cl = (uint32_t *)malloc((w ? w : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < w; ++i) rp[(uint32_t)(pairs[i] >> 32) + 1]++;
    for (uint32_t v = 0; v < nv; ++v) rp[v + 1] += rp[v];
    for (uint64_t i = 0; i < w; ++i) cl[i] = (uint32_t)pairs[i]; /* already sorted */
    free(pairs);

    uint32_t *cnt = (uint32_t *)calloc((size_t)nv, sizeof(uint32_t));
    uint64_t total = 0;
    for (uint32_t a = 0; a < nv; ++a) {
        for (uint32_t j = rp[a]; j < rp[a + 1]; ++j) {
            uint32_t b = cl[j];
            /* merge-intersect N+(a) after b with N+(b) (trianglecounting.cpp:226-246) */
            uint32_t i1 = j + 1, i2 = rp[b];
            uint32_t found = 0;
            while (i1 < rp[a + 1] && i2 < rp[b + 1]) {
                uint32_t x = cl[i1], y = cl[i2];
                if (x == y) { cnt[x]++; ++found; ++i1; ++i2; }
                else if (x < y) ++i1;
                else ++i2;
            }
            cnt[a] += found;
            cnt[b] += found;
            total += found;
        }
    }
    if (per_rank) memcpy(per_rank, cnt, (size_t)nv * sizeof(uint32_t));
    free(cnt); free(rp); free(cl); free(rank);
    return total;
}

/* ---- personalised PageRank --------------------------------------------- */

int orc_ppr(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
            const uint32_t *outdeg, const uint32_t *sources, uint32_t k, double damping,
            int max_sweeps, double tol, float *out) {
    size_t n = (size_t)nv * k;
    float *r = (float *)calloc(n, sizeof(float));
    float *c = (float *)calloc(n, sizeof(float));
    float *acc = (float *)malloc((size_t)k * sizeof(float));
    double *dsum = (double *)malloc((size_t)k * sizeof(double));
    double *nsum = (double *)malloc((size_t)k * sizeof(double));
    int *frozen = (int *)calloc(k, sizeof(int)); /* a source stops after its own first sweep <= tol */
    for (uint32_t s = 0; s < k; ++s) r[(size_t)sources[s] * k + s] = 1.0f;
    int sweeps = 0;
    for (int it = 0; it < max_sweeps; ++it) {
        for (uint32_t v = 0; v < nv; ++v)
            for (uint32_t s = 0; s < k; ++s)
                c[(size_t)v * k + s] = outdeg[v] ? r[(size_t)v * k + s] / (float)outdeg[v] : 0.0f;
        for (uint32_t s = 0; s < k; ++s) { dsum[s] = 0; nsum[s] = 0; }
        for (uint32_t v = 0; v < nv; ++v) {
            for (uint32_t s = 0; s < k; ++s) acc[s] = 0.0f;
            for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) {
                const float *cu = c + (size_t)in_col[j] * k;
                for (uint32_t s = 0; s < k; ++s) acc[s] += cu[s];
            }
            for (uint32_t s = 0; s < k; ++s) {
                if (frozen[s]) continue;
                double tele = (sources[s] == v) ? (1.0 - damping) : 0.0;
                float x = (float)(tele + damping * (double)acc[s]);
                float *rv = r + (size_t)v * k + s;
                dsum[s] += fabs((double)x - (double)*rv);
                nsum[s] += fabs((double)x);
                *rv = x;
            }
        }
        ++sweeps;
        int active = 0;
        for (uint32_t s = 0; s < k; ++s) {
            if (frozen[s]) continue;
            double q = nsum[s] > 0 ? dsum[s] / nsum[s] : 0.0;
            if (tol > 0 && q <= tol) frozen[s] = 1;
            else ++active;
        }
        if (active == 0) break;
    }
    memcpy(out, r, n * sizeof(float));
    free(frozen);
    free(r); free(c); free(acc); free(dsum); free(nsum);
    return sweeps;
}

/* ---- multithreaded variants for full-size checks ----------------------- */

/* The seeded R-MAT generator of the library (csrc/gcg_rng.h), restated: edge i,
 * level l draws u = hi32 (l even) or lo32 (l odd) of
 * SplitMix64(key + (i*ceil(scale/2) + l/2 + 1) * golden), key =
 * SplitMix64(seed ^ 0x6A09E667F3BCC909); u < floor(a 2^32) -> quadrant (0,0),
 * < floor((a+b) 2^32) -> (0,1), < floor((a+b+c) 2^32) -> (1,0), else (1,1); the
 * (src, dst) bits are appended most significant first. Edges are independent,
 * so the threads split them freely. */
static uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

void orc_rmat_edges(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed,
                    uint32_t *src, uint32_t *dst) {
    const double two32 = 4294967296.0;
    const uint64_t ta = (uint64_t)(a * two32), tab = (uint64_t)((a + b) * two32),
                   tabc = (uint64_t)((a + b + c) * two32);
    const uint64_t key = orc_mix64(seed ^ 0x6A09E667F3BCC909ULL);
    const uint64_t ndraw = (scale + 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)m; ++ii) {
        const uint64_t i = (uint64_t)ii;
        uint32_t s = 0, d = 0;
        uint64_t w = 0;
        for (uint32_t l = 0; l < scale; ++l) {
            if ((l & 1u) == 0) w = orc_mix64(key + (i * ndraw + (l >> 1) + 1) * 0x9E3779B97F4A7C15ULL);
            const uint64_t u = (l & 1u) ? (w & 0xFFFFFFFFULL) : (w >> 32);
            const uint32_t q = (u >= ta) + (u >= tab) + (u >= tabc);
            s = (s << 1) | (q >> 1);
            d = (d << 1) | (q & 1u);
        }
        src[i] = s;
        dst[i] = d;
    }
}

#define ORC_BLK 65536u /* rows per residual block: the FP64 sums do not depend on the thread count */

/* orc_pagerank_jacobi with the rows of a sweep split across OpenMP threads.
 * Every row's float sum is the same ascending-source sum, so the ranks are
 * bit-identical to the single-threaded function; the residual's two FP64 sums
 * are formed per block of ORC_BLK rows and the blocks added in order. */
int orc_pagerank_jacobi_mt(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                           const uint32_t *outdeg, double teleport, double damping, float init,
                           int max_sweeps, double tol, float *out_rank, double *res_log) {
    float *r = (float *)malloc((size_t)nv * sizeof(float));
    float *c = (float *)malloc((size_t)nv * sizeof(float));
    float *cn = (float *)malloc((size_t)nv * sizeof(float));
    const uint32_t nb = (nv + ORC_BLK - 1) / ORC_BLK;
    double *part = (double *)malloc(2 * (size_t)(nb ? nb : 1) * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)nv; ++v) {
        r[v] = init;
        c[v] = outdeg[v] ? r[v] / (float)outdeg[v] : 0.0f;
    }
    int sweeps = 0;
    for (int s = 0; s < max_sweeps; ++s) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t bk = 0; bk < (int64_t)nb; ++bk) {
            double dsum = 0, nsum = 0;
            const uint32_t v0 = (uint32_t)bk * ORC_BLK, v1 = v0 + ORC_BLK < nv ? v0 + ORC_BLK : nv;
            for (uint32_t v = v0; v < v1; ++v) {
                float sum = 0.0f;
                for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
                const float x = (float)(teleport + damping * (double)sum);
                dsum += fabs((double)x - (double)r[v]);
                nsum += fabs((double)x);
                r[v] = x;
                cn[v] = outdeg[v] ? x / (float)outdeg[v] : 0.0f;
            }
            part[2 * bk] = dsum;
            part[2 * bk + 1] = nsum;
        }
        double dsum = 0, nsum = 0;
        for (uint32_t bk = 0; bk < nb; ++bk) {
            dsum += part[2 * bk];
            nsum += part[2 * bk + 1];
        }
        float *t = c; c = cn; cn = t;
        ++sweeps;
        const double res = nsum > 0 ? dsum / nsum : 0.0;
        if (res_log) res_log[s] = res;
        if (tol > 0 && res <= tol) break;
    }
    memcpy(out_rank, r, (size_t)nv * sizeof(float));
    free(r); free(c); free(cn); free(part);
    return sweeps;
}

/* orc_pagerank_jacobi_f64 split across OpenMP threads (rows independent, the
 * residual summed per block as above). init_vec (may be NULL) replaces the
 * constant start. res_log (may be NULL) receives each sweep's residual. */
int orc_pagerank_jacobi_f64_mt(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                               const uint32_t *outdeg, double teleport, double damping, double init,
                               const double *init_vec, int max_sweeps, double tol, double *out_rank,
                               double *res_log) {
    double *r = (double *)malloc((size_t)nv * sizeof(double));
    double *c = (double *)malloc((size_t)nv * sizeof(double));
    double *cn = (double *)malloc((size_t)nv * sizeof(double));
    const uint32_t nb = (nv + ORC_BLK - 1) / ORC_BLK;
    double *part = (double *)malloc(2 * (size_t)(nb ? nb : 1) * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)nv; ++v) {
        r[v] = init_vec ? init_vec[v] : init;
        c[v] = outdeg[v] ? r[v] / outdeg[v] : 0.0;
    }
    int sweeps = 0;
    for (int s = 0; s < max_sweeps; ++s) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t bk = 0; bk < (int64_t)nb; ++bk) {
            double dsum = 0, nsum = 0;
            const uint32_t v0 = (uint32_t)bk * ORC_BLK, v1 = v0 + ORC_BLK < nv ? v0 + ORC_BLK : nv;
            for (uint32_t v = v0; v < v1; ++v) {
                double sum = 0.0;
                for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
                const double x = teleport + damping * sum;
                dsum += fabs(x - r[v]);
                nsum += fabs(x);
                r[v] = x;
                cn[v] = outdeg[v] ? x / outdeg[v] : 0.0;
            }
            part[2 * bk] = dsum;
            part[2 * bk + 1] = nsum;
        }
        double dsum = 0, nsum = 0;
        for (uint32_t bk = 0; bk < nb; ++bk) {
            dsum += part[2 * bk];
            nsum += part[2 * bk + 1];
        }
        double *t = c; c = cn; cn = t;
        ++sweeps;
        const double res = nsum > 0 ? dsum / nsum : 0.0;
        if (res_log) res_log[s] = res;
        if (tol > 0 && res <= tol) break;
    }
    memcpy(out_rank, r, (size_t)nv * sizeof(double));
    free(r); free(c); free(cn); free(part);
    return sweeps;
}

/* Stable LSD radix sort of the low `bits` bits of 64-bit keys, 16-bit digits,
 * OpenMP: each thread counts its contiguous block, one thread turns the counts
 * into digit-major / thread-minor offsets, each thread scatters its block.
 * Returns the buffer holding the result (a or tmp). */
static uint64_t *radix_sort_u64_mt(uint64_t *a, uint64_t *tmp, uint64_t n, int bits) {
    const int maxt = omp_get_max_threads();
    uint64_t *cnt = (uint64_t *)malloc((size_t)maxt * 65536 * sizeof(uint64_t));
    uint64_t *src = a, *dst = tmp;
    const int passes = (bits + 15) / 16;
#pragma omp parallel
    {
        const int T = omp_get_num_threads(), t = omp_get_thread_num();
        const uint64_t lo = n * (uint64_t)t / (uint64_t)T, hi = n * (uint64_t)(t + 1) / (uint64_t)T;
        uint64_t *c = cnt + (size_t)t * 65536;
        for (int pass = 0; pass < passes; ++pass) {
            const int sh = 16 * pass;
            memset(c, 0, 65536 * sizeof(uint64_t));
            for (uint64_t i = lo; i < hi; ++i) c[(src[i] >> sh) & 0xFFFF]++;
#pragma omp barrier
#pragma omp single
            {
                uint64_t run = 0;
                for (int d = 0; d < 65536; ++d)
                    for (int u = 0; u < T; ++u) {
                        uint64_t *cu = cnt + (size_t)u * 65536 + d;
                        const uint64_t x = *cu;
                        *cu = run;
                        run += x;
                    }
            }
            for (uint64_t i = lo; i < hi; ++i) dst[c[(src[i] >> sh) & 0xFFFF]++] = src[i];
#pragma omp barrier
#pragma omp single
            {
                uint64_t *x = src;
                src = dst;
                dst = x;
            }
        }
    }
    free(cnt);
    return src;
}

/* The in-CSR of the canonical edge set, for full-size checks: self-loops
 * dropped (sharder.hpp:428-431), duplicates removed, rows by destination with
 * sources ascending -- the same arrays as orc_canonical_edges(dedup) followed by
 * orc_build_csr(by_dst=1), built with a multithreaded radix sort of
 * (dst, src) keys. nv_cap bounds every id (rowptr holds nv_cap+1 entries, col m,
 * outdeg nv_cap). Writes nv = max id + 1 (1 if no edge is left); returns E. */
uint64_t orc_in_csr_mt(const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t nv_cap,
                       uint32_t *nv_out, uint32_t *rowptr, uint32_t *col, uint32_t *outdeg) {
    int vb = 1;
    while (vb < 32 && (1ull << vb) < (uint64_t)nv_cap) ++vb;
    uint64_t *k = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    uint64_t *tmp = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    uint64_t n = 0;
    for (uint64_t i = 0; i < m; ++i) /* sequential: keeps it simple, memory-bound */
        if (src[i] != dst[i]) k[n++] = ((uint64_t)dst[i] << vb) | src[i];
    uint64_t *sorted = radix_sort_u64_mt(k, tmp, n, 2 * vb);
    const uint64_t mask = (1ull << vb) - 1;
    uint64_t E = 0;
    uint32_t maxid = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (i > 0 && sorted[i] == sorted[i - 1]) continue;
        sorted[E++] = sorted[i]; /* in place: E <= i */
    }
    memset(outdeg, 0, (size_t)nv_cap * sizeof(uint32_t));
    for (uint32_t v = 0; v <= nv_cap; ++v) rowptr[v] = 0;
    for (uint64_t i = 0; i < E; ++i) {
        const uint32_t d = (uint32_t)(sorted[i] >> vb), s = (uint32_t)(sorted[i] & mask);
        col[i] = s;
        rowptr[d + 1]++;
        outdeg[s]++;
        if (d > maxid) maxid = d;
        if (s > maxid) maxid = s;
    }
    for (uint32_t v = 0; v < nv_cap; ++v) rowptr[v + 1] += rowptr[v];
    *nv_out = E ? maxid + 1 : 1;
    free(k);
    free(tmp);
    return E;
}

/* Vertex-API PageRank, edge-value program (example_apps/pagerank.cpp:73-113;
 * the app runs it when num_vertices * 4 >= membudget, :166-177) under the
 * engine's deterministic id-ordered execution: sequential Gauss-Seidel in vertex
 * id order where the state lives on the edges. Iteration 0 writes
 * (float)(1.0 / outdeg) to every out-edge and 0.15 to the vertex (:80-85);
 * iteration i >= 1 sums the in-edge values in ascending source order in float
 * (:89-92), pagerank = (float)(0.15 + 0.85 * (double)sum) (:94), writes
 * pagerank / outdeg (float division) to the out-edges (:98-104) and logs
 * |pagerank - old value| (float) into the iteration's delta sum, added in
 * double in vertex order (:108, src/api/graphchi_context.hpp:98-103). Every
 * out-edge of a vertex holds the same value, so one value per source stands for
 * them. out_values = vertex values after niters iterations; delta_log (may be
 * NULL) gets niters entries (entry 0, the initialisation, is 0). */
void orc_pagerank_gs_edge(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                          const uint32_t *outdeg, int niters, float *out_values, double *delta_log) {
    const double RESET = 0.15; /* pagerank.cpp:43 RANDOMRESETPROB */
    float *c = (float *)malloc((size_t)(nv ? nv : 1) * sizeof(float));
    float *val = (float *)malloc((size_t)(nv ? nv : 1) * sizeof(float));
    for (int it = 0; it < niters; ++it) {
        double delta = 0.0;
        for (uint32_t v = 0; v < nv; ++v) {
            const uint32_t outc = outdeg[v];
            if (it == 0) {
                c[v] = outc ? (float)(1.0 / (double)outc) : 0.0f;
                val[v] = (float)RESET;
            } else {
                float sum = 0.0f;
                for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
                const float pagerank = (float)(RESET + (1 - RESET) * (double)sum);
                if (outc > 0) c[v] = pagerank / (float)outc;
                delta += (double)fabsf(pagerank - val[v]);
                val[v] = pagerank;
            }
        }
        if (delta_log) delta_log[it] = delta;
    }
    memcpy(out_values, val, (size_t)nv * sizeof(float));
    free(c);
    free(val);
}

/* Either vertex-API program (edge = 0: in-memory, pagerank.cpp:121-146; edge =
 * 1: edge values, :73-113) in the engine's id order, tracking each vertex's
 * pagerank (float)(0.15 + 0.85 * (double)sum) from sweep to sweep: delta_log[k]
 * = sum of |pagerank - previous| (float differences, added in double in vertex
 * order), res_log[k] = delta_log[k] / sum |pagerank|. The previous value before
 * the first sweep is the vertex value the app holds then: 0.15 for the edge
 * program (:84), pr * outc = 1 (0.15 without out-edges) for the in-memory one
 * (:137-139). Stops after the first sweep whose residual is <= tol (tol > 0) or
 * after max_sweeps; out_values as the app stores them after the last sweep.
 * Returns the sweeps run. */
int orc_pagerank_gs_track(uint32_t nv, const uint32_t *in_rowptr, const uint32_t *in_col,
                          const uint32_t *outdeg, int edge, int max_sweeps, double tol,
                          float *out_values, double *delta_log, double *res_log) {
    const double RESET = 0.15;
    float *c = (float *)malloc((size_t)(nv ? nv : 1) * sizeof(float));
    float *val = (float *)malloc((size_t)(nv ? nv : 1) * sizeof(float));
    for (uint32_t v = 0; v < nv; ++v) {
        const uint32_t outc = outdeg[v];
        if (edge) {
            c[v] = outc ? (float)(1.0 / (double)outc) : 0.0f;
            val[v] = (float)RESET;
        } else {
            c[v] = outc ? 1.0f / (float)outc : (float)RESET;
            val[v] = outc ? 1.0f : (float)RESET;
        }
    }
    int sweeps = 0;
    for (int sw = 0; sw < max_sweeps; ++sw) {
        double dsum = 0.0, nsum = 0.0;
        for (uint32_t v = 0; v < nv; ++v) {
            const uint32_t outc = outdeg[v];
            float sum = 0.0f;
            for (uint32_t j = in_rowptr[v]; j < in_rowptr[v + 1]; ++j) sum += c[in_col[j]];
            const double t = RESET + (1 - RESET) * (double)sum;
            const float pagerank = (float)t;
            if (edge) {
                if (outc > 0) c[v] = pagerank / (float)outc;
            } else {
                c[v] = outc > 0 ? (float)(t / (double)outc) : (float)t;
            }
            dsum += (double)fabsf(pagerank - val[v]);
            nsum += fabs((double)pagerank);
            val[v] = pagerank;
        }
        ++sweeps;
        const double res = nsum > 0 ? dsum / nsum : 0.0;
        if (delta_log) delta_log[sw] = dsum;
        if (res_log) res_log[sw] = res;
        if (tol > 0 && res <= tol) break;
    }
    for (uint32_t v = 0; v < nv; ++v) {
        if (edge) out_values[v] = val[v];
        else out_values[v] = outdeg[v] > 0 ? c[v] * (float)outdeg[v] : c[v];
    }
    free(c);
    free(val);
    return sweeps;
}
