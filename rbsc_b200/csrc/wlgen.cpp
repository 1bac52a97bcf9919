// Seeded generator of the small-graph batch: many small undirected graphs
// (symmetric arcs), half Erdos-Renyi with mean degree about 4 and half random
// 3-regular, with uniform initial labels, concatenated into one CSR over
// global node ids plus the first node of every graph.
//
// Every random draw is a counter-based hash of (seed, graph, purpose, index),
// so a graph does not depend on the thread that builds it or on the other
// graphs, and the batch is the same for any thread count.
//
// Rules (fixed here, the callers and tests rely on them):
//   node count   n = nmin + draw(g, 0, 0) mod (nmax - nmin + 1)
//   graph kind   even g: Erdos-Renyi; odd g: 3-regular
//   Erdos-Renyi  edge {u, v} (u < v) iff draw(g, 2, u*n + v) < 2^64 * 4/(n-1)
//                (every pair when n <= 5)
//   3-regular    n is rounded down to even, and up to 4 if smaller; the
//                pairing model: 3n points sorted by draw(g, 3, attempt*3n + p),
//                consecutive points paired, point p belongs to node p / 3;
//                attempts repeat until the pairing has no loop and no
//                repeated edge
//   labels       1 + draw(g, 1, u) mod num_labels
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/rbsc.h"

rbsc_status rbsc_fail(struct rbsc_ctx* ctx, rbsc_status st, const char* fmt, ...);

namespace {

inline uint64_t fmix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

struct Draw {
    uint64_t base;
    Draw(uint64_t seed, uint64_t g) : base(fmix64(seed + (g + 1) * 0x9E3779B97F4A7C15ull)) {}
    uint64_t operator()(uint32_t tag, uint64_t i) const
    {
        return fmix64(base ^ ((uint64_t)tag << 56) ^ ((i + 1) * 0xD1B54A32D192ED03ull));
    }
};

struct Small {
    uint32_t n = 0;
    std::vector<uint32_t> labels;
    std::vector<uint32_t> off;  // n + 1, local
    std::vector<uint32_t> idx;  // local heads
    bool ok = true;
};

void build_csr(Small& s, std::vector<std::pair<uint32_t, uint32_t>>& edges)
{
    std::vector<std::pair<uint32_t, uint32_t>> arcs;
    arcs.reserve(edges.size() * 2);
    for (auto& e : edges) {
        arcs.emplace_back(e.first, e.second);
        arcs.emplace_back(e.second, e.first);
    }
    std::sort(arcs.begin(), arcs.end());
    s.off.assign(s.n + 1, 0);
    s.idx.resize(arcs.size());
    for (size_t i = 0; i < arcs.size(); ++i) {
        ++s.off[arcs[i].first + 1];
        s.idx[i] = arcs[i].second;
    }
    for (uint32_t u = 0; u < s.n; ++u) s.off[u + 1] += s.off[u];
}

void make_graph(uint64_t seed, uint64_t g, uint32_t nmin, uint32_t nmax, uint32_t num_labels, Small& s)
{
    const Draw d(seed, g);
    uint32_t n = nmin + (uint32_t)(d(0, 0) % (uint64_t)(nmax - nmin + 1));
    const bool regular = (g & 1) != 0;
    if (regular) {
        n &= ~1u;
        n = std::max(n, 4u);
    }
    s.n = n;
    s.labels.resize(n);
    for (uint32_t u = 0; u < n; ++u) s.labels[u] = 1u + (uint32_t)(d(1, u) % num_labels);
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    if (!regular) {
        const unsigned __int128 t = n <= 5 ? ((unsigned __int128)1 << 64) : (((unsigned __int128)4 << 64) / (n - 1));
        const bool all = t >= ((unsigned __int128)1 << 64);
        const uint64_t thr = all ? ~0ull : (uint64_t)t;
        for (uint32_t u = 0; u < n; ++u)
            for (uint32_t v = u + 1; v < n; ++v)
                if (all || d(2, (uint64_t)u * n + v) < thr) edges.emplace_back(u, v);
    } else {
        const uint32_t pts = 3 * n;
        std::vector<std::pair<uint64_t, uint32_t>> key(pts);
        bool done = false;
        for (uint64_t attempt = 0; attempt < 100000 && !done; ++attempt) {
            for (uint32_t p = 0; p < pts; ++p) key[p] = {d(3, attempt * pts + p), p};
            std::sort(key.begin(), key.end());
            edges.clear();
            bool simple = true;
            for (uint32_t k = 0; k < pts && simple; k += 2) {
                uint32_t a = key[k].second / 3, b = key[k + 1].second / 3;
                if (a == b) simple = false;
                if (a > b) std::swap(a, b);
                edges.emplace_back(a, b);
            }
            if (simple) {
                std::sort(edges.begin(), edges.end());
                simple = std::adjacent_find(edges.begin(), edges.end()) == edges.end();
            }
            done = simple;
        }
        if (!done) s.ok = false;
    }
    build_csr(s, edges);
}

}  // namespace

extern "C" rbsc_status rbsc_gen_wl_batch(uint32_t num_graphs, uint32_t nmin, uint32_t nmax, uint32_t num_labels, uint64_t seed,
                                         int32_t threads, rbsc_graph_batch* out)
{
    if (!out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null output");
    std::memset(out, 0, sizeof *out);
    if (num_graphs == 0 || nmin < 2 || nmax < nmin || nmax > 100000 || num_labels == 0)
        return rbsc_fail(nullptr, RBSC_ERR_INVALID, "need num_graphs >= 1, 2 <= nmin <= nmax <= 100000, num_labels >= 1");
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<Small> gs(num_graphs);
    {
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t)
            ts.emplace_back([&, t] {
                for (uint64_t g = (uint64_t)num_graphs * t / threads; g < (uint64_t)num_graphs * (t + 1) / threads; ++g)
                    make_graph(seed, g, nmin, nmax, num_labels, gs[g]);
            });
        for (auto& x : ts) x.join();
    }
    uint64_t n = 0, m = 0;
    for (auto& s : gs) {
        if (!s.ok) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "3-regular pairing did not succeed");
        n += s.n;
        m += s.idx.size();
    }
    if (n >= (1ull << 31)) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "batch too large");
    out->num_graphs = num_graphs;
    out->graph_nodes = (uint64_t*)std::malloc(sizeof(uint64_t) * ((size_t)num_graphs + 1));
    out->labels = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(n, 1));
    out->csr.n = (uint32_t)n;
    out->csr.m = m;
    out->csr.offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * (n + 1));
    out->csr.indices = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(m, 1));
    out->csr.weights = nullptr;
    if (!out->graph_nodes || !out->labels || !out->csr.offsets || !out->csr.indices) {
        rbsc_graph_batch_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    uint64_t nb = 0, mb = 0;
    for (uint32_t g = 0; g < num_graphs; ++g) {
        const Small& s = gs[g];
        out->graph_nodes[g] = nb;
        for (uint32_t u = 0; u < s.n; ++u) {
            out->labels[nb + u] = s.labels[u];
            out->csr.offsets[nb + u] = mb + s.off[u];
        }
        for (size_t i = 0; i < s.idx.size(); ++i) out->csr.indices[mb + i] = (uint32_t)(nb + s.idx[i]);
        nb += s.n;
        mb += s.idx.size();
    }
    out->graph_nodes[num_graphs] = nb;
    out->csr.offsets[nb] = mb;
    return RBSC_OK;
}

extern "C" void rbsc_graph_batch_free(rbsc_graph_batch* b)
{
    if (!b) return;
    std::free(b->graph_nodes);
    std::free(b->labels);
    std::free(b->csr.offsets);
    std::free(b->csr.indices);
    std::free(b->csr.weights);
    std::memset(b, 0, sizeof *b);
}
