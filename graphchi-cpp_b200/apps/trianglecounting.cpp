/*
 * Triangle counting app on the B200 engine: same command line and outputs as
 * example_apps/trianglecounting.cpp (:429-492): <file>.vertexmap (original id
 * -> degree rank), <file>_degord.4B.vout (triangles through each rank) and the
 * line "Number of triangles: T(3T)"; assertequals=N checks the count.
 * The reference refuses nshards=1 (its in-memory mode); the device engine has no
 * such restriction.
 */
#include "graphchi_gpu/graphchi_gpu.hpp"

using namespace graphchi;

struct TriangleCountingProgram : public GraphChiProgram<uint32_t, uint32_t> {
    device_program device_kind() const override { return device_program::triangle_counting; }
};

int main(int argc, const char **argv) {
    try {
        graphchi_init(argc, argv);
        metrics m("triangle-counting");
        std::string filename = get_option_string("file");
        int nshards = convert_if_notexists_novalues<uint32_t>(filename, get_option_string("nshards", "auto"));
        TriangleCountingProgram program;
        graphchi_engine<uint32_t, uint32_t> engine(filename, nshards, true, m);
        engine.run(program, 100000);
        metrics_report(m);
        size_t ntriangles = sum_vertices<vid_t, size_t>(filename + "_degord", 0, (vid_t)engine.num_vertices());
        std::cout << "Number of triangles: " << ntriangles / 3 << "(" << ntriangles << ")" << std::endl;
        size_t expected = get_option_long("assertequals", 0);
        if (expected > 0) {
            std::cout << "Testing the result is as expected: " << (ntriangles / 3) << " vs. " << expected << std::endl;
            if (expected != ntriangles / 3) return 2;
        }
    } catch (const std::exception &e) {
        std::cerr << "trianglecounting: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
