// bvgraph.cpp -- reader of BV-compressed graphs (the WebGraph format of the
// LAW datasets the reference benchmarks on; the reference decodes them with
// its vendored webgraph-rs and pipes them to rbsc as arcs-cuda text, one
// "u 1 v" line per successor v of u: webgraph-rs cli/src/to/arcscuda.rs:61-66).
//
// The format (Boldi & Vigna, "The WebGraph Framework I: Compression
// Techniques", WWW 2004), as far as the default codes go:
//   basename.properties  nodes, arcs, windowsize, minintervallength, zetak,
//                        compressionflags (empty = the default codes below)
//   basename.graph       one bit stream, most significant bit of each byte
//                        first; node x's successor list, for x = 0, 1, ...:
//     outdegree d                      gamma
//     if d > 0 and windowsize > 0:
//       reference r (0..windowsize)    unary; r > 0 copies from node x - r
//       if r > 0: block count b        gamma; then b block lengths, gamma,
//                                      each after the first minus 1; blocks
//                                      alternate copy / skip over the
//                                      referenced list, starting with copy;
//                                      past the last block the rest is copied
//                                      iff b is even
//     if successors remain and minintervallength > 0:
//       interval count c               gamma; interval i: left end (first:
//                                      x + nat2int(gamma), then one past the
//                                      previous interval + 1 + gamma: two
//                                      intervals are never adjacent), length
//                                      (gamma + minintervallength)
//     the remaining successors         zeta_k gaps: first x + nat2int(zeta),
//                                      then previous + 1 + zeta
//   The list is the sorted union of the copied, interval and residual parts.
//   basename.offsets     gamma-coded differences of the bit position where
//                        every node's list starts (used here as a check).
// Codes: unary(n) = n zeros then a one; gamma(n) = unary(l) and the l low
// bits of n + 1, l = floor(log2(n + 1)); zeta_k(n) = unary(h) and h*k + k - 1
// or h*k + k bits (Boldi & Vigna, "Codes for the World Wide Web", 2005);
// nat2int(n) = n / 2 for even n, -(n + 1) / 2 for odd n.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/rbsc.h"

rbsc_status rbsc_fail(struct rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...);

namespace {

bool read_file(const std::string& path, std::vector<uint8_t>& out)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = out.empty() ? 0 : std::fread(out.data(), 1, out.size(), f);
    std::fclose(f);
    return got == out.size();
}

// Bits most significant first; reads past the end give zeros and set `over`.
struct BitReader {
    const uint8_t* p = nullptr;
    uint64_t nbits = 0, pos = 0;
    bool over = false;
    size_t nbytes = 0;

    BitReader(const std::vector<uint8_t>& b) : p(b.data()), nbits(8ull * b.size()), nbytes(b.size()) {}

    // the next 64 bits from `pos`, left-aligned
    uint64_t window() const
    {
        const uint64_t byte = pos >> 3;
        uint64_t w = 0;
        for (int i = 0; i < 9; ++i) {
            const uint64_t b = byte + (uint64_t)i < nbytes ? p[byte + i] : 0u;
            if (i < 8) w = (w << 8) | b;
            else w = (w << (pos & 7)) | (b >> (8 - (pos & 7)));
        }
        return w;
    }
    uint64_t bits(uint32_t n)  // n <= 56
    {
        if (n == 0) return 0;
        const uint64_t v = window() >> (64 - n);
        pos += n;
        if (pos > nbits) over = true;
        return v;
    }
    uint32_t bit() { return (uint32_t)bits(1); }
    uint64_t unary()
    {
        uint64_t z = 0;
        for (;;) {
            const uint64_t w = window();
            if (w) {
                const uint32_t lz = (uint32_t)__builtin_clzll(w);
                z += lz;
                pos += lz + 1;
                break;
            }
            z += 64;
            pos += 64;
            if (pos > nbits) {
                over = true;
                return z;
            }
        }
        if (pos > nbits) over = true;
        return z;
    }
    uint64_t gamma()
    {
        const uint64_t l = unary();
        if (l > 56) {
            over = true;
            return 0;
        }
        return ((1ull << l) | bits((uint32_t)l)) - 1ull;
    }
    uint64_t zeta(uint32_t k)
    {
        const uint64_t h = unary();
        if (h * k + k > 56) {
            over = true;
            return 0;
        }
        const uint64_t left = 1ull << (h * k);
        const uint64_t m = bits((uint32_t)(h * k + k - 1));
        if (m < left) return m + left - 1;
        return (m << 1) + bit() - 1;
    }
};

inline int64_t nat2int(uint64_t n) { return (n & 1) ? -(int64_t)((n + 1) >> 1) : (int64_t)(n >> 1); }

bool parse_properties(const std::string& path, std::map<std::string, std::string>& kv)
{
    std::vector<uint8_t> b;
    if (!read_file(path, b)) return false;
    std::string s(b.begin(), b.end());
    size_t i = 0;
    while (i < s.size()) {
        size_t e = s.find('\n', i);
        if (e == std::string::npos) e = s.size();
        std::string line = s.substr(i, e - i);
        i = e + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty() || line[0] == '#') continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        kv[line.substr(0, eq)] = line.substr(eq + 1);
    }
    return true;
}

}  // namespace

extern "C" rbsc_status rbsc_bv_load(const char* basename, rbsc_host_graph* out, rbsc_bv_stats* stats)
{
    if (!basename || !out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    if (stats) std::memset(stats, 0, sizeof *stats);
    const std::string base(basename);
    std::map<std::string, std::string> kv;
    if (!parse_properties(base + ".properties", kv)) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "cannot read %s.properties", basename);
    auto num = [&](const char* k, uint64_t def, bool need) -> int64_t {
        auto it = kv.find(k);
        if (it == kv.end()) return need ? -1 : (int64_t)def;
        char* end = nullptr;
        const unsigned long long v = std::strtoull(it->second.c_str(), &end, 10);
        return (end && *end == 0) ? (int64_t)v : -1;
    };
    const int64_t nodes = num("nodes", 0, true), arcs = num("arcs", 0, true);
    const int64_t window = num("windowsize", 7, false), minint = num("minintervallength", 4, false);
    const int64_t zk = num("zetak", 3, false);
    if (nodes < 0 || arcs < 0 || window < 0 || minint < 0 || zk <= 0 || zk > 16)
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s.properties: missing or malformed nodes / arcs / codes", basename);
    if (nodes >= 0x80000000ll) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "%lld nodes: must be < 2^31", (long long)nodes);
    auto cf = kv.find("compressionflags");
    if (cf != kv.end() && !cf->second.empty())
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "compression flags \"%s\": only the default codes are supported",
                         cf->second.c_str());
    auto gc = kv.find("graphclass");
    if (gc != kv.end() && gc->second.find("BVGraph") == std::string::npos)
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "graph class %s is not a BVGraph", gc->second.c_str());
    std::vector<uint8_t> gb;
    if (!read_file(base + ".graph", gb)) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "cannot read %s.graph", basename);
    std::vector<uint8_t> ob;
    const bool have_offsets = read_file(base + ".offsets", ob);

    const uint32_t n = (uint32_t)nodes;
    out->n = n;
    out->offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * ((size_t)n + 1));
    out->indices = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<int64_t>(arcs, 1));
    if (!out->offsets || !out->indices) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    BitReader in(gb);
    BitReader offs(ob);
    uint64_t expect_pos = 0;
    uint64_t m = 0, copied_total = 0, interval_total = 0, residual_total = 0;
    std::vector<uint32_t> copied, ivl, res;
    const uint32_t k = (uint32_t)zk;
    auto bad = [&](const char* what, uint32_t x) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s.graph: %s at node %u", basename, what, x);
    };
    for (uint32_t x = 0; x < n; ++x) {
        out->offsets[x] = m;
        if (have_offsets) {
            expect_pos += offs.gamma();
            if (offs.over) return bad("offsets file too short", x);
            if (expect_pos != in.pos) return bad("list does not start at its recorded bit offset", x);
        }
        const uint64_t d = in.gamma();
        if (in.over) return bad("truncated outdegree", x);
        if (d == 0) continue;
        if (m + d > (uint64_t)arcs) return bad("more arcs than the properties declare", x);
        copied.clear();
        ivl.clear();
        res.clear();
        uint64_t extra = d;
        if (window > 0) {
            const uint64_t r = in.unary();
            if (r > (uint64_t)window || r > x) return bad("reference outside the window", x);
            if (r > 0) {
                const uint32_t ref = x - (uint32_t)r;
                const uint64_t rb = out->offsets[ref], re = out->offsets[ref + 1];
                const uint64_t rdeg = re - rb;
                const uint64_t nb = in.gamma();
                uint64_t p = 0;
                for (uint64_t i = 0; i < nb; ++i) {
                    const uint64_t len = in.gamma() + (i == 0 ? 0 : 1);
                    if (p + len > rdeg) return bad("copy blocks beyond the referenced list", x);
                    if ((i & 1) == 0)
                        for (uint64_t j = 0; j < len; ++j) copied.push_back(out->indices[rb + p + j]);
                    p += len;
                }
                if ((nb & 1) == 0)
                    for (uint64_t j = p; j < rdeg; ++j) copied.push_back(out->indices[rb + j]);
                if (copied.size() > d) return bad("more copied successors than the outdegree", x);
                extra = d - copied.size();
            }
        }
        if (extra > 0 && minint > 0) {
            const uint64_t c = in.gamma();
            int64_t end = 0;  // one past the previous interval
            for (uint64_t i = 0; i < c; ++i) {
                const int64_t left = i == 0 ? (int64_t)x + nat2int(in.gamma()) : end + 1 + (int64_t)in.gamma();
                const uint64_t len = in.gamma() + (uint64_t)minint;
                if (len > extra || left < 0 || left + (int64_t)len > (int64_t)n) return bad("interval out of range", x);
                for (uint64_t j = 0; j < len; ++j) ivl.push_back((uint32_t)(left + (int64_t)j));
                end = left + (int64_t)len;
                extra -= len;
            }
        }
        int64_t prev = 0;
        for (uint64_t i = 0; i < extra; ++i) {
            const int64_t v = i == 0 ? (int64_t)x + nat2int(in.zeta(k)) : prev + 1 + (int64_t)in.zeta(k);
            if (v < 0 || v >= (int64_t)n) return bad("residual out of range", x);
            res.push_back((uint32_t)v);
            prev = v;
        }
        if (in.over) return bad("truncated list", x);
        // the sorted union of the three sorted parts
        uint32_t* dst = out->indices + m;
        size_t a = 0, b = 0, c2 = 0;
        for (uint64_t j = 0; j < d; ++j) {
            uint32_t best = 0xffffffffu;
            int which = -1;
            if (a < copied.size() && copied[a] < best) best = copied[a], which = 0;
            if (b < ivl.size() && ivl[b] < best) best = ivl[b], which = 1;
            if (c2 < res.size() && res[c2] < best) best = res[c2], which = 2;
            if (which == 0) ++a;
            else if (which == 1) ++b;
            else ++c2;
            dst[j] = best;
            if (j > 0 && dst[j] <= dst[j - 1]) return bad("successors not strictly increasing", x);
        }
        copied_total += copied.size();
        interval_total += ivl.size();
        residual_total += res.size();
        m += d;
    }
    out->offsets[n] = m;
    out->m = m;
    if (m != (uint64_t)arcs) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: decoded %llu arcs, the properties declare %lld", basename,
                         (unsigned long long)m, (long long)arcs);
    }
    if (stats) {
        stats->copied_arcs = copied_total;
        stats->interval_arcs = interval_total;
        stats->residual_arcs = residual_total;
        stats->offsets_checked = have_offsets ? 1 : 0;
        stats->bits = in.pos;
    }
    return RBSC_OK;
}
