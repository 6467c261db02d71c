/*
 * src/tests/bulksync_functional_test.cpp on the B200 engine: the reference's
 * known-answer test of bulk-synchronous visibility, run by the device functional
 * plug-in (graphchi_gpu/functional_gpu.cuh). In iteration i every gather must see
 * its neighbour's value of iteration i-1, every scatter the value its vertex
 * computed in the iteration it belongs to, and a plus must only ever combine
 * equal values. The reference asserts inside the kernel; here a broken
 * expectation is counted in device memory and the program exits with status 1 if
 * any was. It also reports how many expectations were checked ("checks N") and,
 * like the reference, leaves every vertex's value (niters - 1) in <file>.4B.vout.
 * Command line as the reference test: file=<edge list> niters=<N, default 5>.
 */
#include <cstdio>

#include "graphchi_gpu/functional_gpu.cuh"

using namespace graphchi;

__device__ unsigned long long g_checks = 0;
__device__ unsigned long long g_violations = 0;

GCG_HD inline void expect(bool ok) {
#ifdef __CUDA_ARCH__
    atomicAdd(&g_checks, 1ull);
    if (!ok) atomicAdd(&g_violations, 1ull);
#else
    (void)ok;
#endif
}

struct smoketest_program : public functional_kernel<int, int> {
    GCG_HD int initial_value(graphchi_context &info, vertex_info &myvertex) { return 0; }
    GCG_HD int reset() { return 0; }
    GCG_HD int op_neighborval(graphchi_context &info, vertex_info &myvertex, vid_t nbid, int nbval) {
        expect(nbval == info.iteration - 1);
        return nbval;
    }
    GCG_HD int plus(int curval, int toadd) {
        expect(curval == 0 || toadd == curval);
        return toadd;
    }
    GCG_HD int compute_vertexvalue(graphchi_context &ginfo, vertex_info &myvertex, int nbvalsum) {
        return ginfo.iteration;
    }
    GCG_HD int value_to_neighbor(graphchi_context &info, vertex_info &myvertex, vid_t nbid, int myval) {
        expect(myval == info.iteration);
        return myval;
    }
};

int main(int argc, const char **argv) {
    try {
        graphchi_init(argc, argv);
        metrics m("test-functional");
        std::string filename = get_option_string("file");
        int niters = get_option_int("niters", 5);
        run_functional_unweighted_synchronous<smoketest_program>(filename, niters, m);
        unsigned long long checks = 0, bad = 0;
        if (cudaMemcpyFromSymbol(&checks, g_checks, sizeof(checks)) != cudaSuccess ||
            cudaMemcpyFromSymbol(&bad, g_violations, sizeof(bad)) != cudaSuccess) {
            fprintf(stderr, "bulksync_smoketest: cannot read the device counters\n");
            return 2;
        }
        printf("checks %llu\n", checks);
        if (bad) {
            printf("Smoketest FAILED: %llu of %llu expectations broken\n", bad, checks);
            return 1;
        }
        printf("Smoketest passed successfully! Your system is working!\n");
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "bulksync_smoketest: %s\n", e.what());
        return 2;
    }
}
