/*
 * Host side of the boundary: the edge-list text parser.
 *
 * Replaces convert_edgelist (src/preprocessing/conversions.hpp:210-288), which
 * reads one line at a time with fgets, skips lines starting with '#' or '%',
 * splits on "\t, " with strtok, converts the first two tokens with atoi and
 * ignores a third (the edge value). Here the file is read in one piece and split
 * into byte ranges at line boundaries; host threads parse their ranges into
 * private arrays that are concatenated in file order, so the edge order is the
 * file's. Where the reference asserts (a line with fewer than two tokens) this
 * returns GCG_ERR_FORMAT with the line number. Self-loops are kept here and
 * dropped by the sharder, like the reference's preprocessing_add_edge.
 */
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "gcgpu.h"

namespace gcg {
int fail(int status, const std::string &msg);
}

namespace {

inline bool is_delim(char c) { return c == '\t' || c == ',' || c == ' '; }

/* atoi: optional leading whitespace, sign, decimal digits; stops at the first
 * other character; the int result is converted to the unsigned vertex id. */
inline uint32_t parse_atoi(const char *p, const char *end) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\v' || *p == '\f' || *p == '\r')) ++p;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    uint32_t v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        v = v * 10u + (uint32_t)(*p - '0');
        ++p;
    }
    return neg ? (uint32_t)(0u - v) : v;
}

struct Chunk {
    std::vector<uint32_t> src, dst;
    uint64_t lines = 0;
    uint64_t bad_line = 0; /* 1-based line number within the chunk, 0 = none */
};

/* Parses complete lines in [b, e). */
void parse_range(const char *b, const char *e, Chunk &out) {
    const char *p = b;
    while (p < e) {
        const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
        const char *le = nl ? nl : e;
        ++out.lines;
        if (p < le && (*p == '#' || *p == '%')) {
            p = nl ? nl + 1 : e;
            continue;
        }
        /* first two tokens */
        const char *t[2];
        const char *te[2];
        int nt = 0;
        const char *q = p;
        while (nt < 2) {
            while (q < le && is_delim(*q)) ++q;
            if (q >= le) break;
            t[nt] = q;
            while (q < le && !is_delim(*q)) ++q;
            te[nt] = q;
            ++nt;
        }
        if (nt < 2) {
            if (!out.bad_line) out.bad_line = out.lines;
            p = nl ? nl + 1 : e;
            continue;
        }
        out.src.push_back(parse_atoi(t[0], te[0]));
        out.dst.push_back(parse_atoi(t[1], te[1]));
        p = nl ? nl + 1 : e;
    }
}

int parse_file(const char *path, std::vector<uint32_t> &src, std::vector<uint32_t> &dst) {
    FILE *f = fopen(path, "rb");
    if (!f) return gcg::fail(GCG_ERR_IO, std::string("could not open ") + path);
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)std::max(0L, sz));
    if (sz > 0 && fread(buf.data(), 1, (size_t)sz, f) != (size_t)sz) {
        fclose(f);
        return gcg::fail(GCG_ERR_IO, std::string("short read of ") + path);
    }
    fclose(f);
    const char *base = buf.data();
    const size_t n = buf.size();
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n < (1u << 20)) nt = 1;
    std::vector<size_t> cut(nt + 1, n);
    cut[0] = 0;
    for (unsigned i = 1; i < nt; ++i) {
        size_t c = n * i / nt;
        if (c < cut[i - 1]) c = cut[i - 1];
        const char *nl = c < n ? (const char *)memchr(base + c, '\n', n - c) : nullptr;
        cut[i] = nl ? (size_t)(nl - base) + 1 : n;
    }
    std::vector<Chunk> chunks(nt);
    std::vector<std::thread> th;
    for (unsigned i = 0; i < nt; ++i)
        th.emplace_back([&, i]() { parse_range(base + cut[i], base + cut[i + 1], chunks[i]); });
    for (auto &x : th) x.join();
    uint64_t total = 0, line0 = 0;
    for (auto &c : chunks) {
        if (c.bad_line)
            return gcg::fail(GCG_ERR_FORMAT, std::string(path) + ": line " + std::to_string(line0 + c.bad_line) +
                                                 " is not in the form \"<from>\\t<to>\"");
        line0 += c.lines;
        total += c.src.size();
    }
    src.clear();
    dst.clear();
    src.reserve(total);
    dst.reserve(total);
    for (auto &c : chunks) {
        src.insert(src.end(), c.src.begin(), c.src.end());
        dst.insert(dst.end(), c.dst.begin(), c.dst.end());
    }
    return GCG_OK;
}

}  // namespace

extern "C" {

int gcg_parse_edgelist_file(const char *path, uint32_t *src, uint32_t *dst, uint64_t capacity, uint64_t *m_out) {
    if (!path || !m_out) return gcg::fail(GCG_ERR_INVALID, "gcg_parse_edgelist_file: null argument");
    std::vector<uint32_t> s, d;
    int st = parse_file(path, s, d);
    if (st) return st;
    *m_out = s.size();
    if (!src || !dst) return GCG_OK;
    if (s.size() > capacity) return gcg::fail(GCG_ERR_INVALID, "gcg_parse_edgelist_file: capacity too small");
    memcpy(src, s.data(), s.size() * 4);
    memcpy(dst, d.data(), d.size() * 4);
    return GCG_OK;
}

int gcg_graph_from_edgelist_file(const char *path, uint32_t flags, uint32_t nshards, gcg_graph **out) {
    if (!path || !out) return gcg::fail(GCG_ERR_INVALID, "gcg_graph_from_edgelist_file: null argument");
    std::vector<uint32_t> s, d;
    int st = parse_file(path, s, d);
    if (st) return st;
    return gcg_graph_from_edges(s.data(), d.data(), s.size(), 0, flags, nshards, out);
}

}  // extern "C"
