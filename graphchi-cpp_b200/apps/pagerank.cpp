/*
 * PageRank app on the B200 engine: same command line, outputs and vertex-value
 * file as example_apps/pagerank.cpp (:148-188). As the reference app it picks
 * the in-memory program (pagerank.cpp:121-146, run bit-exactly by
 * gcg_pagerank(GCG_PR_GS_EXACT)) when num_vertices * 4 < membudget_mb, else the
 * edge-value program (pagerank.cpp:73-113, GCG_PR_GS_EDGE, bit-exact, with its
 * <file>.deltalog). Options: file, niters (4), nshards (auto), top (20),
 * membudget_mb (1024); tol > 0 switches to the Jacobi iteration run to that
 * residual; scheduler=1 (with delta_threshold) to selective scheduling. Jacobi
 * and scheduled runs write <file>.deltalog too.
 */
#include "graphchi_gpu/graphchi_gpu.hpp"

using namespace graphchi;

struct PagerankProgram : public GraphChiProgram<float, float> {
    double tol = 0.0, threshold = 0.0;
    bool inmem = true; /* the in-memory program, else the edge-value one */
    device_program device_kind() const override {
        return inmem ? device_program::pagerank_vertex_api : device_program::pagerank_edge_values;
    }
    double tolerance() const override { return tol; }
    double schedule_threshold() const override { return threshold; }
};

int main(int argc, const char **argv) {
    try {
        graphchi_init(argc, argv);
        metrics m("pagerank");
        std::string filename = get_option_string("file");
        int niters = get_option_int("niters", 4);
        int ntop = get_option_int("top", 20);
        int nshards = convert_if_notexists<float>(filename, get_option_string("nshards", "auto"));
        /* scheduler=1: selective scheduling (a vertex whose rank moves by more than
         * delta_threshold of it schedules its out-neighbours); the reference's app
         * runs without it (pagerank.cpp:156) */
        const bool scheduler = get_option_int("scheduler", 0) != 0;
        graphchi_engine<float, float> engine(filename, nshards, scheduler, m);
        PagerankProgram program;
        /* pagerank.cpp:166 */
        program.inmem = engine.num_vertices() * sizeof(float) < (size_t)engine.get_membudget_mb() * 1024L * 1024L;
        if (program.inmem) std::cout << "Running Pagerank by holding vertices in-memory mode!" << std::endl;
        program.tol = atof(get_option_string("tol", "0").c_str());
        program.threshold = atof(get_option_string("delta_threshold", "0.0001").c_str());
        engine.run(program, program.tol > 0 ? get_option_int("niters", 1000) : niters);
        std::vector<vertex_value<float>> top = get_top_vertices<float>(filename, ntop);
        std::cout << "Print top " << ntop << " vertices:" << std::endl;
        for (int i = 0; i < (int)top.size(); i++)
            std::cout << (i + 1) << ". " << top[i].vertex << "\t" << top[i].value << std::endl;
        metrics_report(m);
    } catch (const std::exception &e) {
        std::cerr << "pagerank: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
