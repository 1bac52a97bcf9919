// genhost.cpp -- seeded host generators of the served mix: directed
// Erdos-Renyi graphs and their random lifts (stand-ins for the reference's
// LAW graphs, which need the network).
//
// Every random draw is a counter-based hash of (seed, purpose, row or arc,
// index), so a graph does not depend on the number of threads that build it.
//
// Rules (fixed here; tests and the bench rely on them):
//   Erdos-Renyi  directed G(n, p), p = mean_degree / (n - 1), no self-loops:
//                row u visits the n - 1 candidate heads in increasing order
//                (v = k + (k >= u) for k = 0 .. n-2) by geometric skips
//                floor(log(r) / log(1 - p)) with r = draw(1, u, j) mapped to
//                (0, 1]; rows come out sorted
//   random lift  base = Erdos-Renyi(base_n, mean_degree); node u*L + i for
//                copy i of base node u; base arc e = (u, v) becomes the L arcs
//                (u*L + i, v*L + pi_e(i)), pi_e a Fisher-Yates shuffle with
//                draws draw(2, e, t); row u*L + i lists the heads of its base
//                row's arcs in base order
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
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

inline uint64_t draw(uint64_t seed, uint32_t tag, uint64_t a, uint64_t i)
{
    return fmix64(fmix64(seed ^ ((uint64_t)tag << 58) ^ (a * 0x9E3779B97F4A7C15ull)) + (i + 1) * 0xD1B54A32D192ED03ull);
}

// uniform in (0, 1]
inline double unit(uint64_t r) { return ((double)(r >> 11) + 1.0) * (1.0 / 9007199254740992.0); }

template <typename F>
void parallel_rows(uint64_t n, int threads, F f)
{
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t)
        ts.emplace_back([&, t] {
            for (uint64_t u = n * t / threads; u < n * (t + 1) / threads; ++u) f(u);
        });
    for (auto& x : ts) x.join();
}

// Heads of row u of directed G(n, p); emit(v) for each, increasing.
template <typename E>
void er_row(uint64_t seed, uint32_t n, double p, double lq, uint32_t u, E emit)
{
    if (n < 2 || p <= 0.0) return;
    const uint64_t cand = n - 1;
    if (p >= 1.0) {
        for (uint64_t k = 0; k < cand; ++k) emit((uint32_t)(k + (k >= u)));
        return;
    }
    uint64_t k = 0;
    bool first = true;
    for (uint64_t j = 0;; ++j) {
        const double skip = std::floor(std::log(unit(draw(seed, 1, u, j))) / lq);
        if (skip >= (double)cand) return;
        const uint64_t step = (uint64_t)skip + (first ? 0 : 1);
        first = false;
        k += step;
        if (k >= cand) return;
        emit((uint32_t)(k + (k >= u)));
    }
}

rbsc_status er_build(uint32_t n, double mean_degree, uint64_t seed, int threads, std::vector<uint64_t>& off,
                     std::vector<uint32_t>& idx)
{
    const double p = n > 1 ? std::min(1.0, mean_degree / (double)(n - 1)) : 0.0;
    const double lq = p < 1.0 ? std::log1p(-p) : 0.0;
    off.assign((size_t)n + 1, 0);
    parallel_rows(n, threads, [&](uint64_t u) {
        uint64_t c = 0;
        er_row(seed, n, p, lq, (uint32_t)u, [&](uint32_t) { ++c; });
        off[u + 1] = c;
    });
    for (uint32_t u = 0; u < n; ++u) off[u + 1] += off[u];
    idx.resize(off[n]);
    parallel_rows(n, threads, [&](uint64_t u) {
        uint64_t pos = off[u];
        er_row(seed, n, p, lq, (uint32_t)u, [&](uint32_t v) { idx[pos++] = v; });
    });
    return RBSC_OK;
}

rbsc_status to_host_graph(uint32_t n, uint64_t m, rbsc_host_graph* out)
{
    out->n = n;
    out->m = m;
    out->offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * ((size_t)n + 1));
    out->indices = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(m, 1));
    out->weights = nullptr;
    if (!out->offsets || !out->indices) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    return RBSC_OK;
}

int thread_count(int32_t threads)
{
    return threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
}

}  // namespace

extern "C" rbsc_status rbsc_gen_er_host(uint32_t n, double mean_degree, uint64_t seed, int32_t threads, rbsc_host_graph* out)
{
    if (!out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null output");
    std::memset(out, 0, sizeof *out);
    if (n >= 0x80000000u) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "N must be < 2^31");
    if (!(mean_degree >= 0.0)) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "mean degree must be >= 0");
    std::vector<uint64_t> off;
    std::vector<uint32_t> idx;
    er_build(n, mean_degree, seed, thread_count(threads), off, idx);
    rbsc_status st = to_host_graph(n, idx.size(), out);
    if (st != RBSC_OK) return st;
    std::memcpy(out->offsets, off.data(), sizeof(uint64_t) * off.size());
    if (!idx.empty()) std::memcpy(out->indices, idx.data(), sizeof(uint32_t) * idx.size());
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_gen_lift_host(uint32_t base_n, double mean_degree, uint32_t lift, uint64_t seed, int32_t threads,
                                          rbsc_host_graph* out)
{
    if (!out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null output");
    std::memset(out, 0, sizeof *out);
    if (lift == 0 || lift > 65536) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "lift must be in [1, 65536]");
    if ((uint64_t)base_n * lift >= 0x80000000ull) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "N must be < 2^31");
    const int T = thread_count(threads);
    std::vector<uint64_t> boff;
    std::vector<uint32_t> bidx;
    er_build(base_n, mean_degree, seed, T, boff, bidx);
    const uint32_t n = base_n * lift;
    const uint64_t m = (uint64_t)bidx.size() * lift;
    rbsc_status st = to_host_graph(n, m, out);
    if (st != RBSC_OK) return st;
    uint64_t* off = out->offsets;
    uint32_t* idx = out->indices;
    parallel_rows(base_n, T, [&](uint64_t u) {
        const uint64_t b0 = boff[u], deg = boff[u + 1] - b0;
        for (uint32_t i = 0; i < lift; ++i) off[u * lift + i] = lift * b0 + i * deg;
        std::vector<uint32_t> perm(lift);
        for (uint64_t k = 0; k < deg; ++k) {
            const uint64_t e = b0 + k;
            for (uint32_t i = 0; i < lift; ++i) perm[i] = i;
            for (uint32_t t = lift - 1; t > 0; --t) {
                const uint32_t r = (uint32_t)(draw(seed, 2, e, t) % (uint64_t)(t + 1));
                std::swap(perm[t], perm[r]);
            }
            const uint32_t vbase = bidx[e] * lift;
            for (uint32_t i = 0; i < lift; ++i) idx[lift * b0 + i * deg + k] = vbase + perm[i];
        }
    });
    off[n] = m;
    return RBSC_OK;
}
