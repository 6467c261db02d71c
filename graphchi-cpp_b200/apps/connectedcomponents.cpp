/*
 * Connected components app on the B200 engine: same command line and outputs as
 * example_apps/connectedcomponents.cpp (:154-188): <file>.4B.vout holds the
 * minimum vertex id of each vertex's weakly connected component and
 * analyze_labels writes <file>.components.
 */
#include "graphchi_gpu/graphchi_gpu.hpp"

using namespace graphchi;

struct ConnectedComponentsProgram : public GraphChiProgram<vid_t, vid_t> {
    device_program device_kind() const override { return device_program::connected_components; }
};

int main(int argc, const char **argv) {
    try {
        graphchi_init(argc, argv);
        metrics m("connected-components");
        std::string filename = get_option_string("file");
        int niters = get_option_int("niters", 1000);
        bool scheduler = get_option_int("scheduler", 0) != 0; /* connectedcomponents.cpp:158 */
        int nshards = convert_if_notexists<vid_t>(filename, get_option_string("nshards", "auto"));
        if (get_option_int("onlyresult", 0) == 0) {
            ConnectedComponentsProgram program;
            graphchi_engine<vid_t, vid_t> engine(filename, nshards, scheduler, m);
            engine.run(program, niters);
        }
        m.start_time("label-analysis");
        analyze_labels<vid_t>(filename);
        m.stop_time("label-analysis");
        metrics_report(m);
    } catch (const std::exception &e) {
        std::cerr << "connectedcomponents: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
