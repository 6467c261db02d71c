/*
 * Oracle program (test infrastructure, not product code): a bulk-synchronous
 * (Jacobi) PageRank written against the reference's own functional API and run
 * by the reference's own functional engine, so that the GPU Jacobi mode has a
 * reference-engine counterpart with the same apply formula as the vertex-API app.
 *
 * It is this repository's code compiled against the reference headers
 * (src/api/functional/functional_api.hpp:54-75 kernel contract;
 * src/api/functional/functional_bulksync.hpp:51-169 bulk-sync vertex and proxy;
 * src/engine/functional/functional_engine.hpp:40-123 engine). The runner below
 * uses the same public calls as run_functional_unweighted_synchronous
 * (functional_api.hpp:123-137) and adds an after_iteration() residual stop.
 *
 * Options (reference command-line style, src/util/cmdopts.hpp):
 *   file=<edge list>  filetype=edgelist  niters=<N>  nshards=<auto|P>
 *   teleport=const    apply = 0.15 + 0.85*sum      (example_apps/pagerank.cpp:94)
 *   teleport=pernode  apply = 0.15/N + 0.85*sum    (example_apps/pagerank_functional.cpp:74)
 *   tol=<t>           stop after the iteration whose normalised L1 change
 *                     sum|new-old| / sum|new| (in double) is <= t (0 = off)
 * Prints one line per iteration "residual <iter> <value>" and "iterations <n>".
 * Vertex values land in <file>.4B.vout like every reference app.
 */
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>
#include <cstdlib>

#include "graphchi_basic_includes.hpp"
#include "api/functional/functional_api.hpp"

using namespace graphchi;

static bool g_tconst = true;
static std::vector<float> g_prev;            // previous-iteration vertex values
static double g_delta = 0.0, g_norm = 0.0;  // shared sums (atomic adds: nested OpenMP teams)

struct pr_oracle_kernel : public functional_kernel<float, float> {
    float initial_value(graphchi_context &info, vertex_info &myvertex) {
        g_prev[myvertex.vertexid] = 1.0f;
        return 1.0;
    }
    float reset() { return 0.0; }
    float op_neighborval(graphchi_context &info, vertex_info &myvertex, vid_t nbid, float nbval) {
        return nbval;
    }
    float plus(float curval, float toadd) { return curval + toadd; }
    float compute_vertexvalue(graphchi_context &ginfo, vertex_info &myvertex, float nbvalsum) {
        float v = g_tconst ? (float)(0.15 + 0.85 * nbvalsum)
                           : (float)(0.15 / ginfo.nvertices + 0.85 * nbvalsum);
        double dv = std::fabs((double)v - (double)g_prev[myvertex.vertexid]);
        double nv = std::fabs((double)v);
#pragma omp atomic
        g_delta += dv;
#pragma omp atomic
        g_norm += nv;
        g_prev[myvertex.vertexid] = v;
        return v;
    }
    float value_to_neighbor(graphchi_context &info, vertex_info &myvertex, vid_t nbid, float myval) {
        return myval / myvertex.outdegree;
    }
};

struct pr_oracle_program : public FunctionalProgramProxyBulkSync<pr_oracle_kernel> {
    double tol = 0.0;
    int done_iters = 0;
    void before_iteration(int iteration, graphchi_context &info) {
        g_delta = 0.0;
        g_norm = 0.0;
    }
    void after_iteration(int iteration, graphchi_context &ginfo) {
        done_iters = iteration + 1;
        if (iteration == 0) return;
        double r = g_norm > 0 ? g_delta / g_norm : 0.0;
        std::printf("residual %d %.17g\n", iteration, r);
        if (tol > 0 && r <= tol) ginfo.set_last_iteration(iteration);
    }
};

int main(int argc, const char **argv) {
    graphchi_init(argc, argv);
    metrics m("pr-functional-oracle");
    std::string filename = get_option_string("file");
    int niters = get_option_int("niters", 4);
    g_tconst = get_option_string("teleport", "const") == "const";
    double tol = atof(get_option_string("tol", "0").c_str());

    typedef FunctionalProgramProxyBulkSync<pr_oracle_kernel> proxy_t;
    int nshards = convert_if_notexists<proxy_t::EdgeDataType>(filename, get_option_string("nshards", "auto"));
    functional_engine<proxy_t::VertexDataType, proxy_t::EdgeDataType, proxy_t::fvertex_t>
        engine(filename, nshards, false, m);
    engine.set_modifies_inedges(false);
    engine.set_modifies_outedges(true);
    engine.set_enable_deterministic_parallelism(false);

    g_prev.assign(engine.num_vertices(), 1.0f);

    pr_oracle_program program;
    program.tol = tol;
    engine.run(program, niters);
    std::printf("iterations %d\n", program.done_iters);
    metrics_report(m);
    return 0;
}
