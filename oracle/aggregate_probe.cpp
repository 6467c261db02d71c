/*
 * Oracle program (test infrastructure, not product code): runs the reference's
 * own post-run readers on a vertex-value file, so that the drop-in shim's
 * versions can be pinned to them.
 *
 * It is this repository's code compiled against the reference headers
 * (src/api/vertex_aggregator.hpp:68-127 sum_vertices / foreach_vertices,
 * src/util/labelanalysis.hpp:67-189 analyze_labels). The files it reads are
 * <base>.4B.vout (uint32 values) and <base>.numvertices, as the reference apps
 * leave them.
 *
 *   aggregate_probe sum <base> <fromv> <tov>   prints "sum <value>"
 *   aggregate_probe labels <base>              writes <base>.components
 */
#include <cstdio>
#include <cstdlib>
#include <string>

#include "graphchi_basic_includes.hpp"
#include "util/labelanalysis.hpp"

using namespace graphchi;

int main(int argc, const char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: aggregate_probe sum <base> <fromv> <tov> | labels <base>\n");
        return 2;
    }
    graphchi_init(argc, argv); /* reads <GRAPHCHI_ROOT>/conf/graphchi.cnf, as every reference app */
    const std::string what = argv[1], base = argv[2];
    if (what == "sum" && argc == 5) {
        const vid_t fromv = (vid_t)std::strtoul(argv[3], nullptr, 10);
        const vid_t tov = (vid_t)std::strtoul(argv[4], nullptr, 10);
        const size_t s = sum_vertices<vid_t, size_t>(base, fromv, tov);
        std::printf("sum %zu\n", s);
        return 0;
    }
    if (what == "labels") {
        analyze_labels<vid_t>(base);
        return 0;
    }
    std::fprintf(stderr, "unknown command\n");
    return 2;
}
