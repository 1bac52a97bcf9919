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
// Up to 19 digits cannot overflow; longer tokens (leading zeros, or values
// near 2^64) are re-read with a check per digit.
inline bool read_num(const char*& p, const char* end, uint64_t& out)
{
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    const char* s = p;
    uint64_t v = 0;
    while (p < end && (unsigned)(*p - '0') < 10u) {
        v = v * 10u + (uint64_t)(*p - '0');
        ++p;
    }
    const size_t len = (size_t)(p - s);
    if (len == 0) return false;
    if (len > 19) {
        v = 0;
        for (const char* q = s; q < p; ++q) {
            const uint64_t d = (uint64_t)(*q - '0');
            if (v > (UINT64_MAX - d) / 10) return false;
            v = v * 10 + d;
        }
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

// A run of consecutive arcs with one source.  `at`: first arc (within the
// chunk while parsing, then global); `row_at`: where the run starts inside
// its source's row (a row can span a chunk boundary).
struct Run {
    uint32_t u;
    uint64_t at, cnt, row_at;
};

// One thread's share of the lines.  Heads in input order, written straight
// into the shared heads array at the chunk's line offset (dst, cap lines of
// room); sources as runs; weights only from the first weight other than 1 on
// (earlier ones are 1).
struct Chunk {
    uint32_t* dst = nullptr;  // not owned: a stretch of the heads array
    uint64_t cap = 0;         // lines in the chunk: an upper bound of its arcs
    uint64_t* wt = nullptr;
    uint64_t n = 0;
    std::vector<Run> runs;
    bool ok = true;
    std::string err;
    ~Chunk() { std::free(wt); }
};

uint64_t count_lines(const char* q, const char* e)
{
    uint64_t cap = 1;
    for (const char* r = q; r < e;) {
        const void* nl = std::memchr(r, '\n', (size_t)(e - r));
        if (!nl) break;
        ++cap;
        r = static_cast<const char*>(nl) + 1;
    }
    return cap;
}

void parse_chunk(Chunk& c, const char* q, const char* e, uint64_t N)
{
    const uint64_t cap = c.cap;
    uint64_t cur = UINT64_MAX;
    while (q < e) {
        // skip blank lines
        const char* r = q;
        while (r < e && (*r == ' ' || *r == '\t' || *r == '\r')) ++r;
        if (r < e && *r == '\n') {
            q = r + 1;
            continue;
        }
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
        if (u != cur) {
            if (!c.runs.empty()) c.runs.back().cnt = c.n - c.runs.back().at;
            c.runs.push_back(Run{(uint32_t)u, c.n, 0, 0});
            cur = u;
        }
        if (w != 1 && !c.wt) {
            c.wt = static_cast<uint64_t*>(std::malloc(sizeof(uint64_t) * cap));
            if (!c.wt) {
                c.ok = false;
                c.err = "out of host memory";
                return;
            }
            for (uint64_t i = 0; i < c.n; ++i) c.wt[i] = 1;
        }
        if (c.wt) c.wt[c.n] = w;
        c.dst[c.n++] = (uint32_t)v;
    }
    if (!c.runs.empty()) c.runs.back().cnt = c.n - c.runs.back().at;
}

template <typename F>
void parallel_for(int T, F&& f)
{
    std::vector<std::thread> ts;
    for (int t = 1; t < T; ++t) ts.emplace_back(f, t);
    f(0);
    for (auto& x : ts) x.join();
}

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
    // every chunk parses into its own stretch of one heads array, at its
    // first line's position: input already in source order (the usual case)
    // is then the CSR's heads without a copy
    std::vector<Chunk> ch(T);
    parallel_for(T, [&](int t) { ch[t].cap = count_lines(cut[t], cut[t + 1]); });
    uint64_t lines = 0;
    std::vector<uint64_t> at(T, 0);
    for (int t = 0; t < T; ++t) {
        at[t] = lines;
        lines += ch[t].cap;
    }
    uint32_t* heads = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(lines, 1));
    if (!heads) return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    for (int t = 0; t < T; ++t) ch[t].dst = heads + at[t];
    parallel_for(T, [&](int t) { parse_chunk(ch[t], cut[t], cut[t + 1], N); });
    uint64_t total = 0;
    bool unit = true;
    std::vector<uint64_t> base(T + 1, 0);
    for (int t = 0; t < T; ++t) {
        if (!ch[t].ok) {
            std::free(heads);
            return rbsc_fail(nullptr, ch[t].err == "out of host memory" ? RBSC_ERR_OOM : RBSC_ERR_PARSE, "%s",
                             ch[t].err.c_str());
        }
        base[t] = total;
        total += ch[t].n;
        unit = unit && !ch[t].wt;
    }
    base[T] = total;
    if (total != M) {
        std::free(heads);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "header announces %llu arcs, input holds %llu", (unsigned long long)M,
                         (unsigned long long)total);
    }

    // arcs must be grouped by source: every source starts exactly one run
    // (a run cut by a chunk boundary continues in the next chunk)
    uint64_t* off = (uint64_t*)std::calloc(N + 1, sizeof(uint64_t));
    uint64_t* wt = unit ? nullptr : (uint64_t*)std::malloc(sizeof(uint64_t) * std::max<uint64_t>(M, 1));
    std::vector<uint8_t> seen(N, 0);
    if (!off || (!unit && !wt)) {
        std::free(off); std::free(heads); std::free(wt);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    int64_t prev = -1;
    bool sorted = true;
    for (int t = 0; t < T; ++t)
        for (Run& r : ch[t].runs) {
            r.at += base[t];
            if ((int64_t)r.u == prev) {  // continues the previous chunk's last run
                r.row_at = off[r.u + 1];
                off[r.u + 1] += r.cnt;
                continue;
            }
            if (seen[r.u]) {
                std::free(off); std::free(heads); std::free(wt);
                return rbsc_fail(nullptr, RBSC_ERR_PARSE, "arcs of node %u are not contiguous (input must be grouped by source)", r.u);
            }
            seen[r.u] = 1;
            sorted = sorted && (int64_t)r.u > prev;
            prev = r.u;
            r.row_at = 0;
            off[r.u + 1] = r.cnt;
        }
    for (uint64_t u = 0; u < N; ++u) off[u + 1] += off[u];

    // heads (and weights) to their rows: in source order the input already is
    // the CSR, chunk by chunk (the heads stay where they were parsed; chunks
    // with blank lines left gaps, closed in chunk order, each stretch moving
    // towards the front); otherwise run by run into a new array
    uint32_t* idx = heads;
    if (sorted) {
        for (int t = 0; t < T; ++t)
            if (ch[t].n && heads + base[t] != ch[t].dst) std::memmove(heads + base[t], ch[t].dst, sizeof(uint32_t) * ch[t].n);
    } else {
        idx = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(M, 1));
        if (!idx) {
            std::free(off); std::free(heads); std::free(wt);
            return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
        }
    }
    parallel_for(T, [&](int t) {
        const Chunk& c = ch[t];
        if (sorted) {
            if (wt)
                for (uint64_t i = 0; i < c.n; ++i) wt[base[t] + i] = c.wt ? c.wt[i] : 1u;
            return;
        }
        for (const Run& r : c.runs) {
            const uint64_t from = r.at - base[t], to = off[r.u] + r.row_at;
            std::memcpy(idx + to, c.dst + from, sizeof(uint32_t) * r.cnt);
            if (wt)
                for (uint64_t i = 0; i < r.cnt; ++i) wt[to + i] = c.wt ? c.wt[from + i] : 1u;
        }
    });
    if (!sorted) std::free(heads);
    out->n = (uint32_t)N;
    out->m = M;
    out->offsets = off;
    out->indices = idx;
    out->weights = wt;
    return 0;
}
