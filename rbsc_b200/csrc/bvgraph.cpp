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
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
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
    size_t nbytes = 0;
    bool over = false;

    BitReader(const std::vector<uint8_t>& b, uint64_t start = 0)
        : p(b.data()), nbits(8ull * b.size()), pos(start), nbytes(b.size())
    {
    }

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

struct Params {
    uint32_t n;
    uint64_t arcs;
    uint64_t window, minint;
    uint32_t k;
};

struct Counts {
    uint64_t copied = 0, interval = 0, residual = 0;
};

struct Scratch {
    std::vector<uint32_t> copied, ivl, res;
};

// Node x's successor list from bit `pos`: into `list` (strictly increasing),
// `end` = the bit after it.  ref(r) gives node r's decoded list as
// (pointer, length).  Returns the error text, or nullptr.
template <typename RefFn>
const char* decode_list(const std::vector<uint8_t>& gb, const Params& P, uint32_t x, uint64_t pos, RefFn&& ref,
                        std::vector<uint32_t>& list, Scratch& sc, Counts& cnt, uint64_t& end)
{
    BitReader in(gb, pos);
    list.clear();
    const uint64_t d = in.gamma();
    if (in.over) return "truncated outdegree";
    end = in.pos;
    if (d == 0) return nullptr;
    if (d > P.arcs) return "more arcs than the properties declare";
    sc.copied.clear();
    sc.ivl.clear();
    sc.res.clear();
    uint64_t extra = d;
    if (P.window > 0) {
        const uint64_t r = in.unary();
        if (r > P.window || r > x) return "reference outside the window";
        if (r > 0) {
            const uint32_t* rl = nullptr;
            uint64_t rdeg = 0;
            if (!ref(x - (uint32_t)r, rl, rdeg)) return "reference chain longer than maxrefcount";
            const uint64_t nb = in.gamma();
            uint64_t p = 0;
            for (uint64_t i = 0; i < nb; ++i) {
                const uint64_t len = in.gamma() + (i == 0 ? 0 : 1);
                if (p + len > rdeg) return "copy blocks beyond the referenced list";
                if ((i & 1) == 0) sc.copied.insert(sc.copied.end(), rl + p, rl + p + len);
                p += len;
            }
            if ((nb & 1) == 0) sc.copied.insert(sc.copied.end(), rl + p, rl + rdeg);
            if (sc.copied.size() > d) return "more copied successors than the outdegree";
            extra = d - sc.copied.size();
        }
    }
    if (extra > 0 && P.minint > 0) {
        const uint64_t c = in.gamma();
        int64_t iend = 0;  // one past the previous interval
        for (uint64_t i = 0; i < c; ++i) {
            const int64_t left = i == 0 ? (int64_t)x + nat2int(in.gamma()) : iend + 1 + (int64_t)in.gamma();
            const uint64_t len = in.gamma() + P.minint;
            if (len > extra || left < 0 || left + (int64_t)len > (int64_t)P.n) return "interval out of range";
            for (uint64_t j = 0; j < len; ++j) sc.ivl.push_back((uint32_t)(left + (int64_t)j));
            iend = left + (int64_t)len;
            extra -= len;
        }
    }
    int64_t prev = 0;
    for (uint64_t i = 0; i < extra; ++i) {
        const int64_t v = i == 0 ? (int64_t)x + nat2int(in.zeta(P.k)) : prev + 1 + (int64_t)in.zeta(P.k);
        if (v < 0 || v >= (int64_t)P.n) return "residual out of range";
        sc.res.push_back((uint32_t)v);
        prev = v;
    }
    if (in.over) return "truncated list";
    // the sorted union of the three sorted parts
    list.resize(d);
    size_t a = 0, b = 0, c2 = 0;
    for (uint64_t j = 0; j < d; ++j) {
        uint32_t best = 0xffffffffu;
        int which = -1;
        if (a < sc.copied.size() && sc.copied[a] < best) best = sc.copied[a], which = 0;
        if (b < sc.ivl.size() && sc.ivl[b] < best) best = sc.ivl[b], which = 1;
        if (c2 < sc.res.size() && sc.res[c2] < best) best = sc.res[c2], which = 2;
        if (which == 0) ++a;
        else if (which == 1) ++b;
        else ++c2;
        list[j] = best;
        if (j > 0 && list[j] <= list[j - 1]) return "successors not strictly increasing";
    }
    cnt.copied += sc.copied.size();
    cnt.interval += sc.ivl.size();
    cnt.residual += sc.res.size();
    end = in.pos;
    return nullptr;
}

// One thread's node range [lo, hi): lists written at their CSR offsets.  A
// list referenced from before lo is decoded privately (following its own
// references back at most maxrefcount steps).
struct RangeJob {
    uint32_t lo = 0, hi = 0;
    Counts cnt;
    const char* err = nullptr;
    uint32_t err_node = 0;
};

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
    const int64_t maxref = num("maxrefcount", 0, false);  // 0: not recorded
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
    const Params P{n, (uint64_t)arcs, (uint64_t)window, (uint64_t)minint, (uint32_t)zk};
    out->n = n;
    out->offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * ((size_t)n + 1));
    out->indices = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<int64_t>(arcs, 1));
    if (!out->offsets || !out->indices) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    auto bad = [&](const char* what, uint32_t x) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s.graph: %s at node %u", basename, what, x);
    };
    Counts total;
    uint64_t m = 0, last_bit = 0;
    const int T = (int)std::max(1u, std::thread::hardware_concurrency());
    const bool parallel = have_offsets && maxref > 0 && T > 1 && n >= (1u << 16);
    if (!parallel) {
        // one pass in node order; the offsets file, when present, is a check
        BitReader offs(ob);
        uint64_t expect_pos = 0, pos = 0;
        std::vector<uint32_t> list;
        Scratch sc;
        for (uint32_t x = 0; x < n; ++x) {
            out->offsets[x] = m;
            if (have_offsets) {
                expect_pos += offs.gamma();
                if (offs.over) return bad("offsets file too short", x);
                if (expect_pos != pos) return bad("list does not start at its recorded bit offset", x);
            }
            auto ref = [&](uint32_t r, const uint32_t*& rl, uint64_t& rdeg) {
                rl = out->indices + out->offsets[r];
                rdeg = out->offsets[r + 1] - out->offsets[r];
                return true;
            };
            uint64_t end = 0;
            if (const char* e = decode_list(gb, P, x, pos, ref, list, sc, total, end)) return bad(e, x);
            if (m + list.size() > (uint64_t)arcs) return bad("more arcs than the properties declare", x);
            std::copy(list.begin(), list.end(), out->indices + m);
            m += list.size();
            pos = end;
        }
        last_bit = pos;
    } else {
        // bit position of every list (the offsets file: gamma-coded gaps)
        std::vector<uint64_t> bitpos((size_t)n + 1);
        {
            BitReader offs(ob);
            uint64_t at = 0;
            for (uint32_t x = 0; x < n; ++x) {
                at += offs.gamma();
                if (offs.over) return bad("offsets file too short", x);
                bitpos[x] = at;
            }
            const uint64_t tail = offs.gamma();  // the end of the last list, when recorded
            bitpos[n] = offs.over ? UINT64_MAX : at + tail;
        }
        if (bitpos[0] != 0) return bad("list does not start at its recorded bit offset", 0);
        // outdegrees (the first code of every list), then the CSR offsets
        std::vector<uint64_t> deg((size_t)n);
        std::vector<RangeJob> jobs(T);
        auto run = [&](auto&& fn) {
            std::vector<std::thread> ts;
            for (int t = 1; t < T; ++t) ts.emplace_back(fn, t);
            fn(0);
            for (auto& x : ts) x.join();
        };
        // ranges of about equal bits
        const uint64_t bits_total = bitpos[n] == UINT64_MAX ? 8ull * gb.size() : bitpos[n];
        {
            uint32_t x = 0;
            for (int t = 0; t < T; ++t) {
                jobs[t].lo = x;
                const uint64_t target = bits_total / (uint64_t)T * (uint64_t)(t + 1);
                while (x < n && (t == T - 1 || bitpos[x] < target)) ++x;
                jobs[t].hi = t == T - 1 ? n : x;
            }
        }
        run([&](int t) {
            for (uint32_t x = jobs[t].lo; x < jobs[t].hi; ++x) {
                BitReader in(gb, bitpos[x]);
                deg[x] = in.gamma();
                if (in.over && !jobs[t].err) {
                    jobs[t].err = "truncated outdegree";
                    jobs[t].err_node = x;
                }
            }
        });
        for (int t = 0; t < T; ++t)
            if (jobs[t].err) return bad(jobs[t].err, jobs[t].err_node);
        for (uint32_t x = 0; x < n; ++x) {
            out->offsets[x] = m;
            m += deg[x];
            if (m > (uint64_t)arcs) return bad("more arcs than the properties declare", x);
        }
        out->offsets[n] = m;
        if (m != (uint64_t)arcs) {
            rbsc_host_graph_free(out);
            return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: decoded %llu arcs, the properties declare %lld", basename,
                             (unsigned long long)m, (long long)arcs);
        }
        run([&](int t) {
            RangeJob& J = jobs[t];
            std::unordered_map<uint32_t, std::vector<uint32_t>> before;  // private lists of nodes < lo
            Scratch sc;
            std::vector<uint32_t> list;
            Counts unused;
            // node r's list, decoding the nodes before lo on demand (depth:
            // references followed so far; a list's chain is at most maxrefcount)
            std::function<bool(uint32_t, const uint32_t*&, uint64_t&, int)> get;
            get = [&](uint32_t r, const uint32_t*& rl, uint64_t& rdeg, int depth) -> bool {
                if (r >= J.lo) {
                    rl = out->indices + out->offsets[r];
                    rdeg = out->offsets[r + 1] - out->offsets[r];
                    return true;
                }
                auto it = before.find(r);
                if (it == before.end()) {
                    if (depth > maxref) return false;
                    std::vector<uint32_t> l;
                    Scratch s2;
                    uint64_t end = 0;
                    auto deeper = [&](uint32_t q, const uint32_t*& ql, uint64_t& qd) { return get(q, ql, qd, depth + 1); };
                    if (decode_list(gb, P, r, bitpos[r], deeper, l, s2, unused, end)) return false;
                    it = before.emplace(r, std::move(l)).first;
                }
                rl = it->second.data();
                rdeg = it->second.size();
                return true;
            };
            for (uint32_t x = J.lo; x < J.hi; ++x) {
                auto ref = [&](uint32_t r, const uint32_t*& rl, uint64_t& rdeg) { return get(r, rl, rdeg, 1); };
                uint64_t end = 0;
                const char* e = decode_list(gb, P, x, bitpos[x], ref, list, sc, J.cnt, end);
                uint32_t at = x;
                if (!e && list.size() != deg[x]) e = "outdegree changed between passes";
                // the next list must start where this one ends (reported at
                // the next node, as the one-pass reader does)
                if (!e && x + 1 < n && end != bitpos[x + 1]) {
                    e = "list does not start at its recorded bit offset";
                    at = x + 1;
                }
                if (e) {
                    J.err = e;
                    J.err_node = at;
                    return;
                }
                std::copy(list.begin(), list.end(), out->indices + out->offsets[x]);
                if (x + 1 == n) last_bit = end;
            }
        });
        for (int t = 0; t < T; ++t) {
            if (jobs[t].err) return bad(jobs[t].err, jobs[t].err_node);
            total.copied += jobs[t].cnt.copied;
            total.interval += jobs[t].cnt.interval;
            total.residual += jobs[t].cnt.residual;
        }
        if (n == 0) last_bit = 0;
    }
    out->offsets[n] = m;
    out->m = m;
    if (m != (uint64_t)arcs) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: decoded %llu arcs, the properties declare %lld", basename,
                         (unsigned long long)m, (long long)arcs);
    }
    if (stats) {
        stats->copied_arcs = total.copied;
        stats->interval_arcs = total.interval;
        stats->residual_arcs = total.residual;
        stats->offsets_checked = have_offsets ? 1 : 0;
        stats->bits = last_bit;
    }
    return RBSC_OK;
}
