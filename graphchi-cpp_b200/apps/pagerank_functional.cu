/*
 * example_apps/pagerank_functional.cpp on the B200 engine: the same functional
 * kernel (gather-apply-scatter methods, now marked GCG_HD so the device calls
 * them) run by graphchi_gpu/functional_gpu.cuh. Same command line (file, niters
 * 4, mode semisync|sync, top 20, onlytop) and the same <file>.4B.vout.
 */
#include "graphchi_gpu/functional_gpu.cuh"

using namespace graphchi;

#define RANDOMRESETPROB 0.15

struct pagerank_kernel : public functional_kernel<float, float> {
    GCG_HD float initial_value(graphchi_context &info, vertex_info &myvertex) { return 1.0; }
    GCG_HD float reset() { return 0.0; }
    GCG_HD float op_neighborval(graphchi_context &info, vertex_info &myvertex, vid_t nbid, float nbval) {
        return nbval;
    }
    GCG_HD float plus(float curval, float toadd) { return curval + toadd; }
    GCG_HD float compute_vertexvalue(graphchi_context &ginfo, vertex_info &myvertex, float nbvalsum) {
        return RANDOMRESETPROB / ginfo.nvertices + (1 - RANDOMRESETPROB) * nbvalsum;
    }
    GCG_HD float value_to_neighbor(graphchi_context &info, vertex_info &myvertex, vid_t nbid, float myval) {
        return myval / myvertex.outdegree;
    }
};

int main(int argc, const char **argv) {
    try {
        graphchi_init(argc, argv);
        metrics m("pagerank");
        std::string filename = get_option_string("file");
        int niters = get_option_int("niters", 4);
        bool onlytop = get_option_int("onlytop", 0) != 0;
        int ntop = get_option_int("top", 20);
        std::string mode = get_option_string("mode", "semisync");
        if (!onlytop) {
            if (mode == "semisync") {
                run_functional_unweighted_semisynchronous<pagerank_kernel>(filename, niters, m);
            } else if (mode == "sync") {
                run_functional_unweighted_synchronous<pagerank_kernel>(filename, niters, m);
            } else {
                std::cerr << "Mode needs to be either 'semisync' or 'sync'." << std::endl;
                return 1;
            }
            metrics_report(m);
        }
        std::vector<vertex_value<float>> top = get_top_vertices<float>(filename, ntop);
        std::cout << "Print top 20 vertices: " << std::endl;
        for (int i = 0; i < (int)top.size(); i++)
            std::cout << (i + 1) << ". " << top[i].vertex << "\t" << top[i].value << std::endl;
    } catch (const std::exception &e) {
        std::cerr << "pagerank_functional: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
