/*
 * graphchi_gpu — header-only C++ drop-in for GraphChi's PSW path, running on
 * libgcgpu (include/gcgpu.h).
 *
 * Mirrors the names, argument meaning and file outputs of the reference API that
 * the PageRank / connected components / triangle counting apps use:
 *   graphchi_init, get_option_*           (src/util/cmdopts.hpp:113-250)
 *   metrics, metrics_report               (src/metrics/metrics.hpp:165, graphchi_basic_includes.hpp:65)
 *   convert_if_notexists[_novalues]<ET>   (src/preprocessing/conversions.hpp:728-790)
 *   GraphChiProgram<VT, ET>, graphchi_context (src/api/graphchi_program.hpp:40-88,
 *                                          src/api/graphchi_context.hpp:45-106)
 *   graphchi_engine<VT, ET>::run          (src/engine/graphchi_engine.hpp:148, :718)
 *   get_top_vertices, sum_vertices, analyze_labels (src/util/toplist.hpp:72,
 *                                          src/api/vertex_aggregator.hpp:125, src/util/labelanalysis.hpp:67)
 *
 * What differs: update() bodies cannot run on the device, so a program names
 * the built-in sm_100a vertex program that implements it (device_program()).
 * The engine runs all iterations in one device call; before_iteration(0) and
 * after_iteration(last) are called once around it. Errors throw gcg_error
 * instead of asserting.
 */
#ifndef GRAPHCHI_GPU_HPP
#define GRAPHCHI_GPU_HPP

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gcgpu.h"

/* functions a functional kernel's methods may carry: callable from device code
 * when the including file is compiled by nvcc (graphchi_gpu/functional_gpu.cuh) */
#ifdef __CUDACC__
#define GCG_HD __host__ __device__
#else
#define GCG_HD
#endif

namespace graphchi {

typedef uint32_t vid_t;

struct gcg_error : std::runtime_error {
    int status;
    gcg_error(int st, const std::string &m) : std::runtime_error(m), status(st) {}
};

inline void gcg_check(int st, const char *what) {
    if (st != GCG_OK) throw gcg_error(st, std::string(what) + ": " + gcg_last_error());
}

/* ---- options (cmdopts.hpp: "key value" or "key=value" pairs; --key=value) ---- */
inline std::map<std::string, std::string> &gcg_options() {
    static std::map<std::string, std::string> o;
    return o;
}

inline void graphchi_init(int argc, const char **argv) {
    auto &o = gcg_options();
    for (int i = 1; i < argc; ++i) {
        std::string a(argv[i]);
        while (!a.empty() && a[0] == '-') a.erase(0, 1);
        size_t eq = a.find('=');
        if (eq != std::string::npos) {
            o[a.substr(0, eq)] = a.substr(eq + 1);
        } else if (i + 1 < argc) {
            o[a] = argv[++i];
        }
    }
}

inline std::string get_option_string(const char *name, std::string def) {
    auto &o = gcg_options();
    auto it = o.find(name);
    return it == o.end() ? def : it->second;
}
inline std::string get_option_string(const char *name) {
    auto &o = gcg_options();
    auto it = o.find(name);
    if (it == o.end()) throw gcg_error(GCG_ERR_INVALID, std::string("missing option ") + name);
    return it->second;
}
inline int get_option_int(const char *name, int def) {
    auto s = get_option_string(name, "");
    return s.empty() ? def : atoi(s.c_str());
}
inline uint64_t get_option_long(const char *name, uint64_t def) {
    auto s = get_option_string(name, "");
    return s.empty() ? def : strtoull(s.c_str(), nullptr, 10);
}
inline float get_option_float(const char *name, float def) {
    auto s = get_option_string(name, "");
    return s.empty() ? def : (float)atof(s.c_str());
}

/* ---- metrics: named wall-clock timers and values ---------------------------- */
class metrics {
    std::string name_;
    std::map<std::string, double> acc_, start_;
    std::map<std::string, std::string> vals_;
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
public:
    explicit metrics(std::string n = "default") : name_(std::move(n)) {}
    void start_time(const std::string &k) { start_[k] = now(); }
    void stop_time(const std::string &k) { acc_[k] += now() - start_[k]; }
    void add_time(const std::string &k, double s) { acc_[k] += s; }
    void set(const std::string &k, const std::string &v) { vals_[k] = v; }
    void set(const std::string &k, double v) { vals_[k] = std::to_string(v); }
    double get_time(const std::string &k) const {
        auto it = acc_.find(k);
        return it == acc_.end() ? 0.0 : it->second;
    }
    void report(std::ostream &os) const {
        os << "=== REPORT FOR " << name_ << " ===" << std::endl;
        for (auto &kv : vals_) os << kv.first << ": " << kv.second << std::endl;
        for (auto &kv : acc_) os << kv.first << ": " << kv.second << " s" << std::endl;
    }
};
inline void metrics_report(metrics &m) { m.report(std::cout); }

/* ---- file names (src/api/chifilenames.hpp:65-71, :75-81) -------------------- */
template <typename VT>
inline std::string filename_vertex_data(const std::string &base) {
    return base + "." + std::to_string(sizeof(VT)) + "B.vout";
}
inline std::string filename_intervals(const std::string &base, int nshards) {
    return base + "." + std::to_string(nshards) + ".intervals";
}

/* ---- the device-resident graph registry: one sharded graph per base name ---- */
struct gpu_graph_entry {
    gcg_graph *g = nullptr;
    int nshards = 0;
    ~gpu_graph_entry() { gcg_graph_free(g); }
};
inline std::map<std::string, std::shared_ptr<gpu_graph_entry>> &gpu_graphs() {
    static std::map<std::string, std::shared_ptr<gpu_graph_entry>> r;
    return r;
}

/* sharder.hpp:563-575: nshards "auto" from the memory budget and edge-value size */
inline int auto_nshards(uint64_t nedges, size_t esize, int membudget_mb) {
    double max_shardsize = membudget_mb * 1024. * 1024. / 8;
    return (int)(1 + (nedges * esize / max_shardsize) + 0.5);
}

/* Parses <base> (edge list), shards it on the device and writes the sharder's
 * metadata files. Returns the number of shards. */
inline int gpu_convert(const std::string &base, const std::string &nshards_string, size_t esize,
                       uint32_t flags = GCG_BUILD_DEDUP) {
    auto it = gpu_graphs().find(base);
    if (it != gpu_graphs().end()) return it->second->nshards;
    std::string ft = get_option_string("filetype", "edgelist");
    if (ft != "edgelist")
        throw gcg_error(GCG_ERR_UNSUPPORTED, "filetype " + ft + " is not supported (edgelist only)");
    uint64_t m = 0;
    gcg_check(gcg_parse_edgelist_file(base.c_str(), nullptr, nullptr, 0, &m), "parse");
    std::vector<uint32_t> s(m), d(m);
    gcg_check(gcg_parse_edgelist_file(base.c_str(), s.data(), d.data(), m, &m), "parse");
    int P;
    if (nshards_string.find("auto") != std::string::npos || nshards_string == "0") {
        gcg_graph *probe = nullptr;
        gcg_check(gcg_graph_from_edges(s.data(), d.data(), m, 0, flags | GCG_BUILD_NO_OUT_CSR, 1, &probe),
                  "sharder");
        gcg_graph_info info;
        gcg_graph_get_info(probe, &info);
        gcg_graph_free(probe);
        P = auto_nshards(info.num_edges, esize, get_option_int("membudget_mb", 800));
    } else {
        P = atoi(nshards_string.c_str());
    }
    auto e = std::make_shared<gpu_graph_entry>();
    gcg_check(gcg_graph_from_edges(s.data(), d.data(), m, 0, flags, (uint32_t)std::max(1, P), &e->g), "sharder");
    gcg_graph_info info;
    gcg_graph_get_info(e->g, &info);
    e->nshards = (int)info.nshards;
    gcg_check(gcg_graph_write_metadata(e->g, base.c_str()), "metadata");
    gpu_graphs()[base] = e;
    return e->nshards;
}

/* conversions.hpp:780 / :786 (duplicate edges are removed, as the configs ask) */
template <typename ET>
inline int convert_if_notexists(std::string base, std::string nshards) { return gpu_convert(base, nshards, sizeof(ET)); }
template <typename ET>
inline int convert_if_notexists_novalues(std::string base, std::string nshards) {
    return gpu_convert(base, nshards, sizeof(ET));
}

/* ---- program, context ------------------------------------------------------ */
enum class device_program {
    pagerank_vertex_api,  /* example_apps/pagerank.cpp in-memory program (Gauss-Seidel, bit-exact) */
    pagerank_edge_values, /* example_apps/pagerank.cpp edge-value program (Gauss-Seidel, bit-exact) */
    pagerank_functional,  /* example_apps/pagerank_functional.cpp, mode sync (Jacobi) */
    connected_components, /* example_apps/connectedcomponents.cpp */
    triangle_counting     /* example_apps/trianglecounting.cpp */
};

/* graphchi_context (graphchi_context.hpp:45-106): plain data, so that device
 * code of a functional kernel can read it (the filename is borrowed) */
struct graphchi_context {
    int iteration = 0;
    int num_iterations = 0;
    int last_iteration = -1;
    uint64_t nvertices = 0;
    uint64_t nedges = 0;
    const char *filename = nullptr;
    double last_residual = 0.0;
    double last_deltasum = 0.0; /* sum |change| of the last iteration (graphchi_context::get_delta) */
    GCG_HD void set_last_iteration(int it) { last_iteration = it; }
    GCG_HD double get_delta() const { return last_deltasum; }
};

/* vertex_info of the functional API (functional_defs.hpp:36-40) */
struct vertex_info {
    vid_t vertexid;
    int indegree;
    int outdegree;
};

/* Base of a functional (gather-apply-scatter) kernel (functional_api.hpp:54-75).
 * A kernel defines, with GCG_HD on each so the device can call them:
 *   VT initial_value(graphchi_context&, vertex_info&)           iteration 0
 *   VT reset()                                                   before the gather
 *   ET op_neighborval(graphchi_context&, vertex_info&, vid_t nb, ET nbval)   gather
 *   VT plus(VT curval, ET toadd)                                 sum
 *   VT compute_vertexvalue(graphchi_context&, vertex_info&, VT sum)          apply
 *   ET value_to_neighbor(graphchi_context&, vertex_info&, vid_t nb, VT val)  scatter
 * and runs with run_functional_unweighted_synchronous<KERNEL> from
 * graphchi_gpu/functional_gpu.cuh. The methods are called on the kernel's own type
 * (no virtual dispatch), so the device runs them directly. */
template <typename FVertexDataType, typename FEdgeDataType>
struct functional_kernel {
    typedef FVertexDataType VertexDataType;
    typedef FEdgeDataType EdgeDataType;
};

template <typename VertexDataType, typename EdgeDataType>
struct GraphChiProgram {
    typedef VertexDataType VertexDataType_t;
    virtual ~GraphChiProgram() {}
    virtual void before_iteration(int iteration, graphchi_context &) {}
    virtual void after_iteration(int iteration, graphchi_context &) {}
    virtual void before_exec_interval(vid_t, vid_t, graphchi_context &) {}
    virtual void after_exec_interval(vid_t, vid_t, graphchi_context &) {}
    virtual bool repeat_updates(graphchi_context &) { return false; }
    /* The device vertex program implementing this program's update(). */
    virtual device_program device_kind() const = 0;
    /* Optional convergence tolerance for PageRank (0 = run niters). */
    virtual double tolerance() const { return 0.0; }
    /* With selective scheduling: a PageRank vertex whose value moves by more than
     * this (relative) schedules its out-neighbours (GCG_PR_DELTA). */
    virtual double schedule_threshold() const { return 0.0; }
};

/* ---- engine ---------------------------------------------------------------- */
template <typename VertexDataType, typename EdgeDataType>
class graphchi_engine {
    std::string base_;
    int nshards_;
    metrics &m_;
    graphchi_context ctx_;
    int membudget_mb_;
    bool scheduling_;
    std::shared_ptr<gpu_graph_entry> entry_;

    /* <base>.deltalog, one "iteration,nupdates,work,delta" line per iteration as
     * graphchi_engine::write_delta_log (graphchi_engine.hpp:593-599): cumulative
     * vertex updates and edges processed, the iteration's sum of |change| */
    void write_delta_log(const std::vector<double> &delta, const std::vector<uint64_t> &work, int n) {
        FILE *f = fopen((base_ + ".deltalog").c_str(), "w");
        if (!f) return;
        for (int i = 0; i < n; ++i)
            fprintf(f, "%d,%lu,%lu,%lf\n", i, (unsigned long)work[2 * i], (unsigned long)work[2 * i + 1], delta[i]);
        fclose(f);
    }

    /* The .deltalog the reference's engine writes for the app's vertex programs
     * after `niters` iterations (iteration 0 = initialisation). With one shard and
     * fewer than 80M vertices the engine runs in its in-memory mode
     * (graphchi_engine.hpp:299-301, maxwindow 40M :199) and writes one line after
     * all iterations, with the counters of all of them (:465-506; no edges counted
     * for an adjacency-only program) and every iteration's changes summed;
     * otherwise one line per iteration with cumulative counters (:540-569): vertex
     * updates, and in-edges (in-memory program, out-edges disabled) or in- plus
     * out-edges (edge-value program). delta[i]: the change logged in iteration i
     * (0 for the in-memory program, which calls no log_change). */
    void write_vertex_program_log(bool edge_values, const std::vector<double> &delta, int niters) {
        const uint64_t nv = num_vertices(), ne = num_edges();
        const bool engine_inmem = entry_->nshards == 1 && nv < 2ull * 40000000ull;
        FILE *f = fopen((base_ + ".deltalog").c_str(), "w");
        if (!f) return;
        if (engine_inmem) {
            double d = 0.0;
            for (int i = 0; i < niters; ++i) d += delta[i];
            fprintf(f, "%d,%lu,%lu,%lf\n", niters - 1, (unsigned long)(nv * niters),
                    (unsigned long)(edge_values ? ne * niters : 0), d);
        } else {
            for (int i = 0; i < niters; ++i)
                fprintf(f, "%d,%lu,%lu,%lf\n", i, (unsigned long)(nv * (i + 1)),
                        (unsigned long)((edge_values ? 2 : 1) * ne * (i + 1)), delta[i]);
        }
        fclose(f);
    }

public:
    graphchi_engine(std::string base, int nshards, bool selective_scheduling, metrics &m)
        : base_(std::move(base)), nshards_(nshards), m_(m), membudget_mb_(get_option_int("membudget_mb", 1024)),
          scheduling_(selective_scheduling) {
        auto it = gpu_graphs().find(base_);
        if (it == gpu_graphs().end()) {
            gpu_convert(base_, std::to_string(nshards_ > 0 ? nshards_ : 1), sizeof(EdgeDataType));
            it = gpu_graphs().find(base_);
        }
        entry_ = it->second;
        m_.set("file", base_);
        m_.set("engine", std::string("gcgpu"));
        m_.set("nshards", (double)entry_->nshards);
    }
    /* Setters kept for source compatibility; the device engine has no I/O to tune. */
    void set_modifies_inedges(bool) {}
    void set_modifies_outedges(bool) {}
    void set_only_adjacency(bool) {}
    void set_disable_outedges(bool) {}
    void set_enable_deterministic_parallelism(bool) {}
    void set_exec_threads(int) {}
    void set_load_threads(int) {}
    void set_reset_vertexdata(bool) {}
    void set_membudget_mb(int mb) { membudget_mb_ = mb; }
    int get_membudget_mb() const { return membudget_mb_; }
    gcg_graph *gpu_graph() const { return entry_->g; }

    size_t num_vertices() const {
        gcg_graph_info i;
        gcg_graph_get_info(entry_->g, &i);
        return i.num_vertices;
    }
    size_t num_edges() const {
        gcg_graph_info i;
        gcg_graph_get_info(entry_->g, &i);
        return i.num_edges;
    }
    graphchi_context &get_context() { return ctx_; }

    void run(GraphChiProgram<VertexDataType, EdgeDataType> &program, int niters) {
        m_.start_time("runtime");
        const uint32_t nv = (uint32_t)num_vertices();
        ctx_.filename = base_.c_str();
        ctx_.num_iterations = niters;
        ctx_.nvertices = nv;
        ctx_.nedges = num_edges();
        ctx_.iteration = 0;
        program.before_iteration(0, ctx_);
        std::vector<VertexDataType> values(nv);
        int last = niters - 1;
        switch (program.device_kind()) {
            case device_program::pagerank_vertex_api:
            case device_program::pagerank_edge_values:
            case device_program::pagerank_functional: {
                gcg_pr_params p;
                gcg_pr_params_default(&p);
                const bool edge = program.device_kind() == device_program::pagerank_edge_values;
                const bool vapi = edge || program.device_kind() == device_program::pagerank_vertex_api;
                p.mode = edge ? GCG_PR_GS_EDGE : vapi ? GCG_PR_GS_EXACT : GCG_PR_JACOBI;
                p.max_sweeps = std::max(0, niters - 1);
                p.teleport = vapi ? 0.15 : 0.15 / (double)nv;
                p.tol = program.tolerance();
                if (p.tol > 0) p.mode = GCG_PR_JACOBI;
                if (scheduling_) { /* selective scheduling on the device frontier */
                    p.mode = GCG_PR_DELTA;
                    p.delta_threshold = program.schedule_threshold();
                }
                std::vector<float> r(nv);
                const bool logged = p.mode != GCG_PR_GS_EXACT;
                std::vector<double> dl(logged ? std::max(1, p.max_sweeps) : 0);
                std::vector<uint64_t> wl(logged ? 2 * (size_t)std::max(1, p.max_sweeps) : 0);
                if (logged) {
                    p.delta_log = dl.data();
                    p.work_log = wl.data();
                }
                gcg_pr_stats st;
                gcg_check(gcg_pagerank(entry_->g, &p, r.data(), &st), "pagerank");
                for (uint32_t v = 0; v < nv; ++v) values[v] = (VertexDataType)r[v];
                last = st.sweeps;
                ctx_.last_residual = st.residual;
                if (p.mode == GCG_PR_GS_EDGE || p.mode == GCG_PR_GS_EXACT) {
                    /* iteration 0 (the initialisation) logs no change */
                    std::vector<double> it_delta(1 + (size_t)st.sweeps, 0.0);
                    if (p.mode == GCG_PR_GS_EDGE)
                        for (int i = 0; i < st.sweeps; ++i) it_delta[1 + i] = dl[i];
                    write_vertex_program_log(p.mode == GCG_PR_GS_EDGE, it_delta, st.sweeps + 1);
                    ctx_.last_deltasum = it_delta.back();
                } else if (logged && st.sweeps > 0) {
                    write_delta_log(dl, wl, st.sweeps);
                    ctx_.last_deltasum = dl[st.sweeps - 1];
                }
                m_.add_time("device_sweeps", st.device_ms / 1000.0);
                break;
            }
            case device_program::connected_components: {
                std::vector<uint32_t> lab(nv);
                gcg_cc_stats st;
                if (scheduling_) { /* the reference's label propagation with its scheduler, on a device frontier */
                    gcg_cc_params cp = {GCG_CC_LABEL_PROPAGATION, 1, std::max(1, niters), 0u, nullptr};
                    gcg_check(gcg_connected_components_ex(entry_->g, &cp, lab.data(), &st), "connected components");
                    last = st.passes - 1;
                } else {
                    gcg_check(gcg_connected_components(entry_->g, lab.data(), &st), "connected components");
                }
                for (uint32_t v = 0; v < nv; ++v) values[v] = (VertexDataType)lab[v];
                m_.add_time("device_cc", st.device_ms / 1000.0);
                break;
            }
            case device_program::triangle_counting: {
                std::vector<uint32_t> per(nv), vmap(nv);
                uint64_t total = 0;
                gcg_tc_stats st;
                gcg_check(gcg_triangle_count(entry_->g, &total, per.data(), vmap.data(), &st), "triangle counting");
                /* <base>.vertexmap (orderbydegree.hpp:94-100) and the per-rank counts of <base>_degord */
                std::ofstream vm(base_ + ".vertexmap", std::ios::binary);
                vm.write((const char *)vmap.data(), (std::streamsize)nv * 4);
                gcg_check(gcg_write_vout((base_ + "_degord").c_str(), per.data(), nv, 4), "write vout");
                for (uint32_t v = 0; v < nv; ++v) values[v] = (VertexDataType)per[v];
                m_.add_time("device_tc", st.device_ms / 1000.0);
                break;
            }
        }
        ctx_.iteration = last;
        program.after_iteration(last, ctx_);
        if (program.device_kind() != device_program::triangle_counting)
            gcg_check(gcg_write_vout(base_.c_str(), values.data(), nv, sizeof(VertexDataType)), "write vout");
        m_.stop_time("runtime");
    }
};

/* ---- result readers -------------------------------------------------------- */
template <typename VT>
struct vertex_value {
    vid_t vertex;
    VT value;
};

template <typename VT>
inline std::vector<VT> read_vertex_values(const std::string &base) {
    std::ifstream f(filename_vertex_data<VT>(base), std::ios::binary | std::ios::ate);
    if (!f) throw gcg_error(GCG_ERR_IO, "cannot read " + filename_vertex_data<VT>(base));
    size_t n = (size_t)f.tellg() / sizeof(VT);
    std::vector<VT> v(n);
    f.seekg(0);
    f.read((char *)v.data(), (std::streamsize)(n * sizeof(VT)));
    return v;
}

/* toplist.hpp:72: the ntop largest values, ties by vertex id */
template <typename VT>
inline std::vector<vertex_value<VT>> get_top_vertices(std::string base, int ntop) {
    auto v = read_vertex_values<VT>(base);
    std::vector<vertex_value<VT>> all(v.size());
    for (size_t i = 0; i < v.size(); ++i) all[i] = {(vid_t)i, v[i]};
    size_t k = std::min((size_t)ntop, all.size());
    std::partial_sort(all.begin(), all.begin() + k, all.end(), [](const vertex_value<VT> &a, const vertex_value<VT> &b) {
        return a.value > b.value || (a.value == b.value && a.vertex < b.vertex);
    });
    all.resize(k);
    return all;
}

/* vertex_aggregator.hpp:68-127: the sum over [fromv, tov) read in windows of
 * 2^20 vertices. As in the reference, a window holding a single vertex is
 * skipped (its `if (st < en)` test, :84), so when (tov - fromv) % 2^20 == 1 the
 * last vertex is not added. */
template <typename VT, typename ST>
inline ST sum_vertices(std::string base, vid_t fromv, vid_t tov) {
    auto v = read_vertex_values<VT>(base);
    const vid_t window = 1024 * 1024;
    ST acc = 0;
    for (uint64_t st = fromv; st <= (uint64_t)tov; st += window) {
        uint64_t en = st + window - 1;
        if (en >= (uint64_t)tov) en = (uint64_t)tov - 1;
        if (!(st < en)) continue;
        for (uint64_t i = st; i <= en && i < v.size(); ++i) acc += (ST)v[i];
    }
    return acc;
}

/* labelanalysis.hpp:67-189: component sizes written to <base>.components as
 * "label,size" lines. As in the reference: a vertex whose value is its own id
 * (a component's representative) is not counted, every other vertex adds one
 * to its label, a label's size is printed as count + 1, and labels are listed in
 * decreasing count order as std::sort leaves them when started from ascending
 * label order (so a component of one vertex does not appear). */
template <typename VT>
inline void analyze_labels(std::string base, int printtop = 20) {
    auto v = read_vertex_values<VT>(base);
    uint64_t nv = v.size();
    {
        std::ifstream nf(base + ".numvertices");
        uint64_t x = 0;
        if (nf >> x && x < nv) nv = x;
    }
    struct labelcount {
        VT label;
        uint64_t count;
    };
    std::vector<VT> lab;
    lab.reserve(nv);
    for (uint64_t i = 0; i < nv; ++i)
        if (v[i] != (VT)i && v[i] != VT(0xffffffff)) lab.push_back(v[i]);
    std::sort(lab.begin(), lab.end());
    std::vector<labelcount> cur;
    for (size_t i = 0; i < lab.size(); ++i) {
        if (i > 0 && lab[i] == lab[i - 1]) cur.back().count++;
        else cur.push_back({lab[i], 1});
    }
    std::sort(cur.begin(), cur.end(), [](const labelcount &a, const labelcount &b) { return a.count > b.count; });
    const std::string outname = base + ".components";
    std::ofstream f(outname);
    if (!f) throw gcg_error(GCG_ERR_IO, "cannot write " + outname);
    for (auto &c : cur) f << c.label << "," << c.count + 1 << "\n";
    std::cout << "Total number of different labels (components/communities): " << cur.size() << std::endl;
    std::cout << "List of labels was written to file: " << outname << std::endl;
    for (int i = 0; i < printtop && i < (int)cur.size(); ++i)
        std::cout << (i + 1) << ". label: " << cur[i].label << ", size: " << cur[i].count + 1 << std::endl;
}

}  // namespace graphchi

#endif
