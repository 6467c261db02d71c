// Test helper: runs the drop-in shim's post-run readers (graphchi_gpu.hpp) on a
// vertex-value file, the same way the oracle's aggregate_probe runs the
// reference's. Compiled and run by tests/test_shim_readers.py.
//   shim_readers sum <base> <fromv> <tov>   prints "sum <value>"
//   shim_readers labels <base>              writes <base>.components
#include <cstdio>
#include <cstdlib>
#include <string>

#include "graphchi_gpu/graphchi_gpu.hpp"

int main(int argc, char **argv) {
    if (argc < 3) return 2;
    const std::string what = argv[1], base = argv[2];
    if (what == "sum" && argc == 5) {
        const graphchi::vid_t a = (graphchi::vid_t)std::strtoul(argv[3], nullptr, 10);
        const graphchi::vid_t b = (graphchi::vid_t)std::strtoul(argv[4], nullptr, 10);
        std::printf("sum %zu\n", graphchi::sum_vertices<graphchi::vid_t, size_t>(base, a, b));
        return 0;
    }
    if (what == "labels") {
        graphchi::analyze_labels<graphchi::vid_t>(base);
        return 0;
    }
    return 2;
}
