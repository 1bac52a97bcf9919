// gen.cu -- synthetic workloads standing in for the reference's LAW graphs
// (the reference pipes BV-compressed LAW graphs through webgraph-rs; those
// are not available here).  R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004):
// every arc descends `scale` levels of the adjacency matrix, choosing a
// quadrant with probabilities (a, b, c, d).  Each (arc, level) draw is a hash
// of (seed, arc, level), so the host and device generators produce the same
// graph bit for bit.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "radix.cuh"
#include "scan.cuh"

using namespace rbsc;

namespace {

struct RmatParams {
    uint64_t seed;
    uint32_t scale;
    uint32_t ta, tab, tabc;  // quadrant thresholds scaled to 2^32
};

__host__ __device__ __forceinline__ uint64_t rmat_key(const RmatParams& p, uint64_t e)
{
    const uint64_t base = fmix64(p.seed ^ (e * kGolden));
    uint64_t u = 0, v = 0;
    for (uint32_t l = 0; l < p.scale; ++l) {
        const uint32_t r = (uint32_t)(fmix64(base + (uint64_t)(l + 1) * 0xd1b54a32d192ed03ull) >> 32);
        const uint32_t ub = r >= p.tab ? 1u : 0u;
        const uint32_t vb = ((r >= p.ta && r < p.tab) || r >= p.tabc) ? 1u : 0u;
        u = (u << 1) | ub;
        v = (v << 1) | vb;
    }
    return (u << p.scale) | v;
}

uint32_t thr(double x)
{
    if (x <= 0) return 0;
    const double t = x * 4294967296.0;
    return t >= 4294967295.0 ? 0xffffffffu : (uint32_t)t;
}

RmatParams make_params(uint32_t scale, double a, double b, double c, uint64_t seed)
{
    RmatParams p;
    p.seed = seed;
    p.scale = scale;
    p.ta = thr(a);
    p.tab = thr(a + b);
    p.tabc = thr(a + b + c);
    return p;
}

__global__ void k_rmat_keys(RmatParams p, uint64_t m0, unsigned long long* __restrict__ keys)
{
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m0; e += (uint64_t)gridDim.x * blockDim.x)
        keys[e] = rmat_key(p, e);
}

// keep the first of every run of equal keys, drop self-loops
__global__ void k_rmat_keep(uint64_t m0, uint32_t scale, const unsigned long long* __restrict__ keys, uint32_t* __restrict__ keep)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m0) return;
    const uint64_t k = keys[i];
    const uint64_t mask = (1ull << scale) - 1ull;
    keep[i] = ((i == 0 || keys[i - 1] != k) && ((k >> scale) != (k & mask))) ? 1u : 0u;
}

// Writes the heads of the kept arcs and the CSR offsets, from the sorted keys:
// the first kept arc of source u sits at pos[i] for the first i with src >= u,
// so the thread of key i writes off[x] for every x in (src(i-1), src(i)].
__global__ void k_rmat_emit(uint64_t m0, uint32_t scale, const unsigned long long* __restrict__ keys,
                            const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, uint32_t* __restrict__ idx,
                            uint64_t* __restrict__ off)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m0) return;
    const uint64_t mask = (1ull << scale) - 1ull;
    const uint64_t n = 1ull << scale;
    const uint64_t u = i < m0 ? (keys[i] >> scale) : n;   // i == m0: sentinel past the last source
    const int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> scale);
    for (int64_t x = prev + 1; x <= (int64_t)u && x <= (int64_t)n; ++x) off[x] = pos[i];
    if (i < m0 && keep[i]) idx[pos[i]] = (uint32_t)(keys[i] & mask);
}

// The first `hb` levels of an arc's descent fix the top hb bits of its
// source: the bucket an arc belongs to is known before the remaining levels.
__device__ __forceinline__ uint32_t rmat_src_top(const RmatParams& p, uint64_t base, uint32_t hb)
{
    uint32_t u = 0;
    for (uint32_t l = 0; l < hb; ++l) {
        const uint32_t r = (uint32_t)(fmix64(base + (uint64_t)(l + 1) * 0xd1b54a32d192ed03ull) >> 32);
        u = (u << 1) | (r >= p.tab ? 1u : 0u);
    }
    return u;
}

// Histogram of the arcs over the top hb bits of their source.
__global__ void k_rmat_src_hist(RmatParams p, uint64_t m0, uint32_t hb, unsigned long long* __restrict__ hist)
{
    extern __shared__ unsigned int s_hist[];
    const uint32_t bins = 1u << hb;
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m0; e += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&s_hist[rmat_src_top(p, fmix64(p.seed ^ (e * kGolden)), hb)], 1u);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
}

// Keys of the arcs whose source's top bits fall in [lo, hi), appended.
__global__ void __launch_bounds__(256) k_rmat_bucket_keys(RmatParams p, uint64_t m0, uint32_t hb, uint32_t lo, uint32_t hi,
                                                          unsigned long long* __restrict__ keys, uint32_t* __restrict__ count)
{
    __shared__ BlockReserveSmem<256> sm;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base_e = (uint64_t)blockIdx.x * blockDim.x; base_e < m0; base_e += stride) {
        const uint64_t e = base_e + threadIdx.x;
        bool take = false;
        if (e < m0) {
            const uint32_t top = rmat_src_top(p, fmix64(p.seed ^ (e * kGolden)), hb);
            take = top >= lo && top < hi;
        }
        const uint32_t pos = block_reserve<256>(take, count, sm);
        if (take) keys[pos] = rmat_key(p, e);
    }
}

// Heads of the kept arcs of a bucket (sorted keys) into idx, and the offsets
// of the bucket's sources [s_lo, s_hi): off[x - s_lo] = arc_base + first kept
// arc of source x.
__global__ void k_rmat_bucket_emit(uint64_t mb, uint32_t scale, uint64_t s_lo, uint64_t s_hi, uint64_t arc_base,
                                   const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ keep,
                                   const uint32_t* __restrict__ pos, uint32_t* __restrict__ idx, uint64_t* __restrict__ off)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > mb) return;
    const uint64_t mask = (1ull << scale) - 1ull;
    const uint64_t u = i < mb ? (keys[i] >> scale) : s_hi;  // sentinel past the bucket's last source
    const int64_t prev = i == 0 ? (int64_t)s_lo - 1 : (int64_t)(keys[i - 1] >> scale);
    for (int64_t x = prev + 1; x <= (int64_t)u && x < (int64_t)s_hi; ++x) off[x - s_lo] = arc_base + pos[i];
    if (i < mb && keep[i]) idx[pos[i]] = (uint32_t)(keys[i] & mask);
}

}  // namespace

#define CKG(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) { st = rbsc_cuda_fail(ctx, e_, #call, __LINE__); goto done; } \
    } while (0)
#define CKGS(call)                             \
    do {                                       \
        st = (call);                           \
        if (st != RBSC_OK) goto done;          \
    } while (0)

extern "C" rbsc_status rbsc_gen_rmat_device(rbsc_ctx* ctx, uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                            uint64_t seed, rbsc_graph** out)
{
    if (!ctx || !out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (scale < 1 || scale > 30) return rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "scale must be in [1, 30]");
    const uint64_t n = 1ull << scale;
    const uint64_t m0 = (uint64_t)edge_factor << scale;
    if (m0 >= (1ull << 32)) return rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "device R-MAT generator: edge_factor * 2^scale must be < 2^32");
    rbsc_status st = RBSC_OK;
    cudaStream_t s = ctx->stream;
    unsigned long long *keys0 = nullptr, *keys1 = nullptr;
    uint32_t *keep = nullptr, *pos = nullptr;
    void* tmp = nullptr;
    rbsc_graph* g = nullptr;
    const RmatParams p = make_params(scale, a, b, c, seed);
    const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div<uint64_t>(m0, 256), (uint64_t)ctx->sm_count * 64);
    bool alt = false;
    uint32_t mu = 0;
    const unsigned long long* sorted = nullptr;
    CKG(cudaSetDevice(ctx->device));
    CKGS(dev_alloc(ctx, (void**)&keys0, 8 * m0));
    CKGS(dev_alloc(ctx, (void**)&keys1, 8 * m0));
    CKGS(dev_alloc(ctx, &tmp, std::max(radix_temp_bytes(m0), scan_temp_bytes<uint64_t>(m0 + 1)) + 1024));
    ++rbsc::launch_counter();
    k_rmat_keys<<<grid, 256, 0, s>>>(p, m0, keys0);
    CKG(cudaGetLastError());
    CKG(radix_sort<uint32_t>(keys0, keys1, (uint32_t*)nullptr, (uint32_t*)nullptr, m0, 0, 2 * (int)scale, tmp, s, &alt));
    sorted = alt ? keys1 : keys0;
    CKGS(dev_alloc(ctx, (void**)&keep, 4 * (m0 + 1)));
    CKGS(dev_alloc(ctx, (void**)&pos, 4 * (m0 + 1)));
    ++rbsc::launch_counter();
    k_rmat_keep<<<(unsigned)ceil_div<uint64_t>(m0, 256), 256, 0, s>>>(m0, scale, sorted, keep);
    CKG(cudaGetLastError());
    CKG((exclusive_scan<uint32_t, uint32_t>(keep, pos, m0, pos + m0, tmp, s)));
    CKG(cudaMemcpyAsync(&mu, pos + m0, 4, cudaMemcpyDeviceToHost, s));
    CKG(cudaStreamSynchronize(s));
    g = new rbsc_graph();
    g->ctx = ctx;
    g->n = (uint32_t)n;
    g->m = mu;
    CKGS(graph_alloc_csr(ctx, g, false));
    ++rbsc::launch_counter();
    k_rmat_emit<<<(unsigned)ceil_div<uint64_t>(m0 + 1, 256), 256, 0, s>>>(m0, scale, sorted, keep, pos, g->d_idx, g->d_off);
    CKG(cudaGetLastError());
    CKG(cudaStreamSynchronize(s));
    dev_free(ctx, (void*&)keys0);
    dev_free(ctx, (void*&)keys1);
    dev_free(ctx, (void*&)keep);
    dev_free(ctx, (void*&)pos);
    dev_free(ctx, tmp);
    CKGS(graph_prepare(ctx, g));
    *out = g;
    g = nullptr;
done:
    cudaStreamSynchronize(s);
    dev_free(ctx, (void*&)keys0);
    dev_free(ctx, (void*&)keys1);
    dev_free(ctx, (void*&)keep);
    dev_free(ctx, (void*&)pos);
    dev_free(ctx, tmp);
    if (g) rbsc_graph_free(g);
    return st;
}

// ---------------------------------------------------------------------------
// device generator into page-locked host memory, in source buckets
// ---------------------------------------------------------------------------
extern "C" rbsc_status rbsc_gen_rmat_pinned(rbsc_ctx* ctx, uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                            uint64_t seed, rbsc_host_graph* out)
{
    if (!ctx || !out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    if (scale < 1 || scale > 30) return rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "scale must be in [1, 30]");
    const uint64_t n = 1ull << scale;
    const uint64_t m0 = (uint64_t)edge_factor << scale;
    const uint32_t hb = std::min<uint32_t>(scale, 12);
    const uint32_t bins = 1u << hb;
    const RmatParams p = make_params(scale, a, b, c, seed);
    cudaStream_t s = ctx->stream;
    rbsc_status st = RBSC_OK;
    unsigned long long *hist = nullptr, *keys0 = nullptr, *keys1 = nullptr;
    uint32_t *keep = nullptr, *pos = nullptr, *cnt = nullptr, *didx = nullptr;
    uint64_t* doff = nullptr;
    void* tmp = nullptr;
    std::vector<unsigned long long> h(bins);
    uint64_t cap = 0, arcs = 0;
    const unsigned grid = (unsigned)ctx->sm_count * 16;
    CKG(cudaSetDevice(ctx->device));
    // page-locked output: offsets, and heads for up to m0 arcs (duplicates removed later)
    CKG(cudaHostAlloc((void**)&out->offsets, 8 * (n + 1), cudaHostAllocDefault));
    CKG(cudaHostAlloc((void**)&out->indices, 4 * std::max<uint64_t>(m0, 1), cudaHostAllocDefault));
    out->n = (uint32_t)n;
    CKGS(dev_alloc(ctx, (void**)&hist, 8 * bins));
    CKG(cudaMemsetAsync(hist, 0, 8 * bins, s));
    ++rbsc::launch_counter();
    k_rmat_src_hist<<<grid, 256, 4 * bins, s>>>(p, m0, hb, hist);
    CKG(cudaGetLastError());
    CKG(cudaMemcpyAsync(h.data(), hist, 8 * bins, cudaMemcpyDeviceToHost, s));
    CKG(cudaStreamSynchronize(s));
    // buckets of consecutive bins with at most `cap` arcs (at least one bin)
    cap = std::max<uint64_t>(*std::max_element(h.begin(), h.end()), std::min<uint64_t>(m0, 1ull << 29));
    if (cap > (1ull << 31)) {
        st = rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "R-MAT: %llu arcs share the top %u source bits (limit 2^31)",
                       (unsigned long long)cap, hb);
        goto done;
    }
    CKGS(dev_alloc(ctx, (void**)&keys0, 8 * cap));
    CKGS(dev_alloc(ctx, (void**)&keys1, 8 * cap));
    CKGS(dev_alloc(ctx, (void**)&keep, 4 * (cap + 1)));
    CKGS(dev_alloc(ctx, (void**)&pos, 4 * (cap + 1)));
    CKGS(dev_alloc(ctx, (void**)&didx, 4 * cap));
    CKGS(dev_alloc(ctx, (void**)&doff, 8 * n));
    CKGS(dev_alloc(ctx, (void**)&cnt, 16));
    CKGS(dev_alloc(ctx, &tmp, std::max(radix_temp_bytes(cap), scan_temp_bytes<uint32_t>(cap + 1)) + 1024));
    for (uint32_t lo = 0; lo < bins;) {
        uint32_t hi = lo + 1;
        uint64_t kb = h[lo];
        while (hi < bins && kb + h[hi] <= cap) kb += h[hi++];
        uint32_t mb = 0;
        CKG(cudaMemsetAsync(cnt, 0, 4, s));
        ++rbsc::launch_counter();
        k_rmat_bucket_keys<<<grid, 256, 0, s>>>(p, m0, hb, lo, hi, keys0, cnt);
        CKG(cudaGetLastError());
        CKG(cudaMemcpyAsync(&mb, cnt, 4, cudaMemcpyDeviceToHost, s));
        CKG(cudaStreamSynchronize(s));
        bool alt = false;
        CKG(radix_sort<uint32_t>(keys0, keys1, (uint32_t*)nullptr, (uint32_t*)nullptr, mb, 0, 2 * (int)scale, tmp, s, &alt));
        const unsigned long long* sorted = alt ? keys1 : keys0;
        uint32_t mu = 0;
        if (mb) {
            ++rbsc::launch_counter();
            k_rmat_keep<<<(unsigned)ceil_div<uint64_t>(mb, 256), 256, 0, s>>>(mb, scale, sorted, keep);
            CKG(cudaGetLastError());
            CKG((exclusive_scan<uint32_t, uint32_t>(keep, pos, mb, pos + mb, tmp, s)));
            CKG(cudaMemcpyAsync(&mu, pos + mb, 4, cudaMemcpyDeviceToHost, s));
            CKG(cudaStreamSynchronize(s));
        } else {
            CKG(cudaMemsetAsync(pos, 0, 4, s));
        }
        const uint64_t s_lo = (uint64_t)lo << (scale - hb), s_hi = (uint64_t)hi << (scale - hb);
        ++rbsc::launch_counter();
        k_rmat_bucket_emit<<<(unsigned)ceil_div<uint64_t>((uint64_t)mb + 1, 256), 256, 0, s>>>(mb, scale, s_lo, s_hi, arcs, sorted,
                                                                                              keep, pos, didx, doff);
        CKG(cudaGetLastError());
        if (mu) CKG(cudaMemcpyAsync(out->indices + arcs, didx, 4 * (size_t)mu, cudaMemcpyDeviceToHost, s));
        CKG(cudaMemcpyAsync(out->offsets + s_lo, doff, 8 * (s_hi - s_lo), cudaMemcpyDeviceToHost, s));
        CKG(cudaStreamSynchronize(s));
        arcs += mu;
        lo = hi;
    }
    out->offsets[n] = arcs;
    out->m = arcs;
done:
    cudaStreamSynchronize(s);
    dev_free(ctx, (void*&)hist);
    dev_free(ctx, (void*&)keys0);
    dev_free(ctx, (void*&)keys1);
    dev_free(ctx, (void*&)keep);
    dev_free(ctx, (void*&)pos);
    dev_free(ctx, (void*&)didx);
    dev_free(ctx, (void*&)doff);
    dev_free(ctx, (void*&)cnt);
    dev_free(ctx, tmp);
    if (st != RBSC_OK) rbsc_host_graph_free_pinned(out);
    return st;
}

extern "C" void rbsc_host_graph_free_pinned(rbsc_host_graph* g)
{
    if (!g) return;
    if (g->offsets) cudaFreeHost(g->offsets);
    if (g->indices) cudaFreeHost(g->indices);
    if (g->weights) cudaFreeHost(g->weights);
    std::memset(g, 0, sizeof *g);
}

// ---------------------------------------------------------------------------
// host generator (same arcs as the device one)
// ---------------------------------------------------------------------------
static void host_radix_sort(std::vector<uint64_t>& a, int bits, int threads)
{
    std::vector<uint64_t> b(a.size());
    const size_t n = a.size();
    const int R = 11;
    const size_t B = 1u << R;
    threads = std::max(1, threads);
    std::vector<std::vector<size_t>> cnt(threads, std::vector<size_t>(B));
    for (int shift = 0; shift < bits; shift += R) {
        auto chunk = [&](int t) { return std::make_pair(n * t / threads, n * (t + 1) / threads); };
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t)
            ts.emplace_back([&, t] {
                auto [lo, hi] = chunk(t);
                std::fill(cnt[t].begin(), cnt[t].end(), 0);
                for (size_t i = lo; i < hi; ++i) ++cnt[t][(a[i] >> shift) & (B - 1)];
            });
        for (auto& x : ts) x.join();
        size_t run = 0;
        for (size_t d = 0; d < B; ++d)
            for (int t = 0; t < threads; ++t) {
                const size_t c = cnt[t][d];
                cnt[t][d] = run;
                run += c;
            }
        ts.clear();
        for (int t = 0; t < threads; ++t)
            ts.emplace_back([&, t] {
                auto [lo, hi] = chunk(t);
                for (size_t i = lo; i < hi; ++i) b[cnt[t][(a[i] >> shift) & (B - 1)]++] = a[i];
            });
        for (auto& x : ts) x.join();
        a.swap(b);
    }
}

extern "C" rbsc_status rbsc_gen_rmat_host(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                                          int32_t threads, rbsc_host_graph* out)
{
    if (!out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null output");
    std::memset(out, 0, sizeof *out);
    if (scale < 1 || scale > 30) return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "scale must be in [1, 30]");
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const uint64_t n = 1ull << scale;
    const uint64_t m0 = (uint64_t)edge_factor << scale;
    const RmatParams p = make_params(scale, a, b, c, seed);
    std::vector<uint64_t> keys;
    try {
        keys.resize(m0);
    } catch (...) {
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    {
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t)
            ts.emplace_back([&, t] {
                for (uint64_t e = m0 * t / threads; e < m0 * (t + 1) / threads; ++e) keys[e] = rmat_key(p, e);
            });
        for (auto& x : ts) x.join();
    }
    host_radix_sort(keys, 2 * (int)scale, threads);
    const uint64_t mask = n - 1;
    uint64_t mu = 0;
    for (uint64_t i = 0; i < m0; ++i)
        if ((i == 0 || keys[i - 1] != keys[i]) && ((keys[i] >> scale) != (keys[i] & mask))) ++mu;
    out->n = (uint32_t)n;
    out->m = mu;
    out->offsets = (uint64_t*)std::calloc(n + 1, sizeof(uint64_t));
    out->indices = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(mu, 1));
    out->weights = nullptr;
    if (!out->offsets || !out->indices) {
        std::free(out->offsets);
        std::free(out->indices);
        std::memset(out, 0, sizeof *out);
        return rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
    }
    uint64_t j = 0;
    for (uint64_t i = 0; i < m0; ++i) {
        const uint64_t k = keys[i];
        if ((i == 0 || keys[i - 1] != k) && ((k >> scale) != (k & mask))) {
            out->indices[j++] = (uint32_t)(k & mask);
            ++out->offsets[(k >> scale) + 1];
        }
    }
    for (uint64_t u = 0; u < n; ++u) out->offsets[u + 1] += out->offsets[u];
    return RBSC_OK;
}

extern "C" void rbsc_host_graph_free(rbsc_host_graph* g)
{
    if (!g) return;
    std::free(g->offsets);
    std::free(g->indices);
    std::free(g->weights);
    std::memset(g, 0, sizeof *g);
}
