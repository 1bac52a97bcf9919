// parse.cpp -- arcs-cuda text reader (replaces read_uint64 / read_graph,
// src/rbsc/rbsc.cu:156-180).
//
// Format (webgraph-rs cli/src/to/arcscuda.rs:61-66): "N\nM\n" then M lines
// "u wt v" with the arcs grouped by u.  The reference reader loops forever on
// end of input without a trailing newline and trusts every byte; this one is
// multi-threaded and rejects malformed input with RBSC_ERR_PARSE.  Groups may
// come in any order of u (the reference's ReduceByKey only needs contiguous
// runs); the CSR keeps each row's arcs in input order.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rbsc.h"

rbsc_status rbsc_fail(struct rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...);

namespace {

inline bool is_space(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

// Reads one decimal number; returns false on a missing or malformed token.
inline bool read_num(const char*& p, const char* end, uint64_t& out)
{
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (p >= end || *p < '0' || *p > '9') return false;
    uint64_t v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        const uint64_t d = (uint64_t)(*p - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
        ++p;
    }
    if (p < end && !is_space(*p)) return false;
    out = v;
    return true;
}

inline bool end_line(const char*& p, const char* end)
{
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (p < end && *p != '\n') return false;
    if (p < end) ++p;
    return true;
}

struct Chunk {
    std::vector<uint32_t> src, dst;
    std::vector<uint64_t> wt;
    bool ok = true;
    bool unit = true;
    std::string err;
};

}  // namespace

extern "C" rbsc_status rbsc_parse_arcs(const char* text, size_t len, rbsc_host_graph* out)
{
    if (!out || (!text && len)) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    const char* p = text;
    const char* end = text + len;
    uint64_t N = 0, M = 0;
    while (p < end && is_space(*p)) ++p;
    if (!read_num(p, end, N) || !end_line(p, end)) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "line 1: expected the node count");
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (!read_num(p, end, M) || !end_line(p, end)) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "line 2: expected the arc count");
    if (N >= 0x80000000ull) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "N = %llu: node ids must be < 2^31", (unsigned long long)N);

    // split the body at line starts
    const size_t body = (size_t)(end - p);
    int T = (int)std::max(1u, std::thread::hardware_concurrency());
    if (body < (1u << 20)) T = 1;
    std::vector<const char*> cut(T + 1);
    cut[0] = p;
    cut[T] = end;
    for (int t = 1; t < T; ++t) {
        const char* q = p + body * t / T;
        if (q < cut[t - 1]) q = cut[t - 1];
        while (q < end && *(q - 1) != '\n') ++q;
        cut[t] = q;
    }
    std::vector<Chunk> ch(T);
    std::vector<std::thread> ts;
    for (int t = 0; t < T; ++t)
        ts.emplace_back([&, t] {
            Chunk& c = ch[t];
            const char* q = cut[t];
            const char* e = cut[t + 1];
            while (q < e) {
                // skip blank lines
                const char* r = q;
                while (r < e && (*r == ' ' || *r == '\t' || *r == '\r')) ++r;
                if (r < e && *r == '\n') { q = r + 1; continue; }
                if (r >= e) break;
                uint64_t u, w, v;
                if (!read_num(q, e, u) || !read_num(q, e, w) || !read_num(q, e, v) || !end_line(q, e)) {
                    c.ok = false;
                    c.err = "malformed arc line";
                    return;
                }
                if (u >= N || v >= N) {
                    c.ok = false;
                    c.err = "node id out of range";
                    return;
                }
                c.src.push_back((uint32_t)u);
                c.dst.push_back((uint32_t)v);
                c.wt.push_back(w);
                if (w != 1) c.unit = false;
            }
        });
    for (auto& x : ts) x.join();
    uint64_t total = 0;
    bool unit = true;
    for (auto& c : ch) {
        if (!c.ok) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s", c.err.c_str());
        total += c.src.size();
        unit = unit && c.unit;
    }
    if (total != M)
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "header announces %llu arcs, input holds %llu", (unsigned long long)M,
                         (unsigned long long)total);

    // arcs must be grouped by source: every source starts exactly one run
    std::vector<uint8_t> seen(N, 0);
    uint64_t* off = (uint64_t*)std::calloc(N + 1, sizeof(uint64_t));
    uint32_t* idx = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(M, 1));
    uint64_t* wt = unit ? nullptr : (uint64_t*)std::malloc(sizeof(uint64_t) * std::max<uint64_t>(M, 1));
    if (!off || !idx || (!unit && !wt)) {
        std::free(off); std::free(idx); std::free(wt);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    int64_t prev = -1;
    for (auto& c : ch)
        for (size_t i = 0; i < c.src.size(); ++i) {
            const uint32_t u = c.src[i];
            if ((int64_t)u != prev) {
                if (seen[u]) {
                    std::free(off); std::free(idx); std::free(wt);
                    return rbsc_fail(nullptr, RBSC_ERR_PARSE, "arcs of node %u are not contiguous (input must be grouped by source)", u);
                }
                seen[u] = 1;
                prev = u;
            }
            ++off[u + 1];
        }
    for (uint64_t u = 0; u < N; ++u) off[u + 1] += off[u];
    std::vector<uint64_t> fill(off, off + N);
    for (auto& c : ch)
        for (size_t i = 0; i < c.src.size(); ++i) {
            const uint64_t k = fill[c.src[i]]++;
            idx[k] = c.dst[i];
            if (wt) wt[k] = c.wt[i];
        }
    out->n = (uint32_t)N;
    out->m = M;
    out->offsets = off;
    out->indices = idx;
    out->weights = wt;
    return 0;
}
