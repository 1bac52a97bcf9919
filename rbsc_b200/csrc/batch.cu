// Batches of small graphs: the graphs are refined together as one resident
// graph (their disjoint union, so the colours form one namespace), then the
// per-graph results are taken out of the union's colouring on the device:
//
//   key(u) = (graph of u) << 32 | colour(u)   for every node, value u
//   stable radix sort by key                  -> nodes grouped by graph, then
//                                                by colour, then by node id
//   segment heads + exclusive scan            -> one histogram entry per
//                                                (graph, colour): its colour,
//                                                first position, smallest node
//   per entry                                 -> count, graph fingerprint
//   per node                                  -> local canonical label
//
// A graph's local canonical label of u is the smallest node of u's block in
// u's graph (minus the graph's first node): the same label a refinement of
// that graph alone gives, since the union's coarsest stable partition
// restricted to one graph is that graph's own coarsest stable partition.
#include <algorithm>
#include <chrono>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "common.cuh"
#include "radix.cuh"
#include "scan.cuh"
#include "internal.h"

using namespace rbsc;

namespace {

// graph of node u: the largest i with graph_nodes[i] <= u
__global__ void k_batch_keys(uint32_t n, const uint64_t* __restrict__ gn, uint32_t G, const uint32_t* __restrict__ col,
                             unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    uint32_t lo = 0, hi = G - 1;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo + 1) >> 1);
        if (gn[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    keys[u] = ((unsigned long long)lo << 32) | col[u];
    vals[u] = u;
}

__global__ void k_batch_heads(uint32_t n, const unsigned long long* __restrict__ keys, uint32_t* __restrict__ head)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// One histogram entry per segment of equal keys.  ex = exclusive scan of the
// heads; entry of sorted position i = ex[i] + head[i] - 1.
__global__ void k_batch_entries(uint32_t n, const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                                const uint32_t* __restrict__ head, const uint32_t* __restrict__ ex,
                                uint32_t* __restrict__ ecolor, uint32_t* __restrict__ estart, uint32_t* __restrict__ emin,
                                uint64_t* __restrict__ hoff)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    const uint32_t e = ex[i];
    const unsigned long long k = keys[i];
    ecolor[e] = (uint32_t)k;
    estart[e] = i;
    emin[e] = vals[i];  // the sort is stable and the values started in node order
    const uint32_t g = (uint32_t)(k >> 32);
    if (i == 0 || (uint32_t)(keys[i - 1] >> 32) != g) hoff[g] = e;
}

// Entry counts and the per-graph fingerprint: the sum over its entries of a
// mix of (colour, count), which does not depend on the order of the entries.
__global__ void k_batch_counts(uint32_t H, uint32_t n, const uint32_t* __restrict__ estart, const uint32_t* __restrict__ ecolor,
                               const unsigned long long* __restrict__ keys, uint32_t* __restrict__ ecount,
                               unsigned long long* __restrict__ fp)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= H) return;
    const uint32_t s = estart[e];
    const uint32_t c = (e + 1 < H ? estart[e + 1] : n) - s;
    ecount[e] = c;
    const uint32_t g = (uint32_t)(keys[s] >> 32);
    atomicAdd(&fp[g], (unsigned long long)fmix64(((uint64_t)ecolor[e] << 32 | c) * kGolden + 0x2545f4914f6cdd1dull));
}

__global__ void k_batch_local(uint32_t n, const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                              const uint32_t* __restrict__ head, const uint32_t* __restrict__ ex,
                              const uint32_t* __restrict__ emin, const uint64_t* __restrict__ gn, uint32_t* __restrict__ local)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t e = ex[i] + head[i] - 1u;
    const uint32_t g = (uint32_t)(keys[i] >> 32);
    local[vals[i]] = emin[e] - (uint32_t)gn[g];
}

__global__ void k_batch_blocks(uint32_t G, const uint64_t* __restrict__ hoff, uint32_t* __restrict__ blocks)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) blocks[g] = (uint32_t)(hoff[g + 1] - hoff[g]);
}

unsigned grid_of(uint64_t n) { return (unsigned)std::max<uint64_t>(1, (n + 255) / 256); }

}  // namespace

#define BK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) { st = rbsc_cuda_fail(ctx, e_, #call, __LINE__); goto done; } \
    } while (0)
#define BKS(call)                              \
    do {                                       \
        st = (call);                           \
        if (st != RBSC_OK) goto done;          \
    } while (0)

extern "C" rbsc_status rbsc_graph_batch_refine(rbsc_ctx* ctx, rbsc_graph* g, const uint64_t* graph_nodes, uint32_t num_graphs,
                                               const uint32_t* init_colors, rbsc_batch_result* out, rbsc_stats* stats)
{
    if (!ctx || !g || !graph_nodes || !out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    if (num_graphs == 0) return rbsc_fail(ctx, RBSC_ERR_INVALID, "empty batch");
    if (graph_nodes[0] != 0 || graph_nodes[num_graphs] != g->n)
        return rbsc_fail(ctx, RBSC_ERR_INVALID, "graph_nodes must start at 0 and end at N");
    for (uint32_t i = 0; i < num_graphs; ++i)
        if (graph_nodes[i + 1] <= graph_nodes[i]) return rbsc_fail(ctx, RBSC_ERR_INVALID, "graph %u has no node", i);
    rbsc_status st = RBSC_OK;
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n, G = num_graphs;
    int gbits = 0;
    while (gbits < 32 && (1ull << gbits) < G) ++gbits;
    unsigned long long *keys = nullptr, *keys2 = nullptr, *fp = nullptr;
    uint32_t *vals = nullptr, *vals2 = nullptr, *head = nullptr, *ex = nullptr, *ecolor = nullptr, *estart = nullptr,
             *emin = nullptr, *ecount = nullptr, *local = nullptr, *blocks = nullptr;
    uint64_t* gn = nullptr;
    uint64_t* hoff = nullptr;
    void* tmp = nullptr;
    bool alt = false;
    uint32_t H = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float batch_ms = 0.f;
    // the refinement of the union
    BKS(rbsc_graph_refine(ctx, g, init_colors, out->colors, stats));
    BK(cudaEventCreate(&e0));
    BK(cudaEventCreate(&e1));
    BK(cudaEventRecord(e0, s));
    BKS(dev_alloc(ctx, (void**)&gn, 8 * ((size_t)G + 1)));
    BKS(dev_alloc(ctx, (void**)&keys, 8 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&keys2, 8 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&vals, 4 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&vals2, 4 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&head, 4 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&ex, 4 * ((size_t)n + 1)));
    BKS(dev_alloc(ctx, &tmp, std::max(radix_temp_bytes(n), scan_temp_bytes<uint32_t>((uint64_t)n + 1)) + 1024));
    BK(cudaMemcpyAsync(gn, graph_nodes, 8 * ((size_t)G + 1), cudaMemcpyHostToDevice, s));
    ++rbsc::launch_counter();
    k_batch_keys<<<grid_of(n), 256, 0, s>>>(n, gn, G, g->d_out, keys, vals);
    BK(cudaGetLastError());
    BK(radix_sort<uint32_t>(keys, keys2, vals, vals2, n, 0, 32 + gbits, tmp, s, &alt));
    if (alt) {
        std::swap(keys, keys2);
        std::swap(vals, vals2);
    }
    ++rbsc::launch_counter();
    k_batch_heads<<<grid_of(n), 256, 0, s>>>(n, keys, head);
    BK(cudaGetLastError());
    BK((exclusive_scan<uint32_t, uint32_t>(head, ex, n, ex + n, tmp, s)));
    BK(cudaMemcpyAsync(&H, ex + n, 4, cudaMemcpyDeviceToHost, s));
    BK(cudaStreamSynchronize(s));
    // entries reuse the second sort buffers (free after the sort)
    ecolor = vals2;
    estart = reinterpret_cast<uint32_t*>(keys2);
    emin = estart + n;
    BKS(dev_alloc(ctx, (void**)&ecount, 4 * ((size_t)H + 1)));
    BKS(dev_alloc(ctx, (void**)&hoff, 8 * ((size_t)G + 1)));
    BKS(dev_alloc(ctx, (void**)&fp, 8 * (size_t)G));
    BKS(dev_alloc(ctx, (void**)&local, 4 * (size_t)n));
    BKS(dev_alloc(ctx, (void**)&blocks, 4 * (size_t)G));
    BK(cudaMemsetAsync(fp, 0, 8 * (size_t)G, s));
    {
        const uint64_t hH = H;
        BK(cudaMemcpyAsync(hoff + G, &hH, 8, cudaMemcpyHostToDevice, s));
    }
    ++rbsc::launch_counter();
    k_batch_entries<<<grid_of(n), 256, 0, s>>>(n, keys, vals, head, ex, ecolor, estart, emin, hoff);
    ++rbsc::launch_counter();
    k_batch_counts<<<grid_of(H), 256, 0, s>>>(H, n, estart, ecolor, keys, ecount, fp);
    ++rbsc::launch_counter();
    k_batch_local<<<grid_of(n), 256, 0, s>>>(n, keys, vals, head, ex, emin, gn, local);
    ++rbsc::launch_counter();
    k_batch_blocks<<<grid_of(G), 256, 0, s>>>(G, hoff, blocks);
    BK(cudaGetLastError());
    BK(cudaEventRecord(e1, s));
    if (out->local) BK(cudaMemcpyAsync(out->local, local, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    if (out->blocks) BK(cudaMemcpyAsync(out->blocks, blocks, 4 * (size_t)G, cudaMemcpyDeviceToHost, s));
    if (out->fingerprint) BK(cudaMemcpyAsync(out->fingerprint, fp, 8 * (size_t)G, cudaMemcpyDeviceToHost, s));
    if (out->hist_offsets) BK(cudaMemcpyAsync(out->hist_offsets, hoff, 8 * ((size_t)G + 1), cudaMemcpyDeviceToHost, s));
    if (out->hist_colors) BK(cudaMemcpyAsync(out->hist_colors, ecolor, 4 * (size_t)H, cudaMemcpyDeviceToHost, s));
    if (out->hist_counts) BK(cudaMemcpyAsync(out->hist_counts, ecount, 4 * (size_t)H, cudaMemcpyDeviceToHost, s));
    BK(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&batch_ms, e0, e1);
    if (stats) {
        stats->device_ms += batch_ms;
        stats->time_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
done:
    cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    dev_free(ctx, (void*&)gn);
    dev_free(ctx, (void*&)keys);
    dev_free(ctx, (void*&)keys2);
    dev_free(ctx, (void*&)vals);
    dev_free(ctx, (void*&)vals2);
    dev_free(ctx, (void*&)head);
    dev_free(ctx, (void*&)ex);
    dev_free(ctx, tmp);
    dev_free(ctx, (void*&)ecount);
    dev_free(ctx, (void*&)hoff);
    dev_free(ctx, (void*&)fp);
    dev_free(ctx, (void*&)local);
    dev_free(ctx, (void*&)blocks);
    return st;
}

extern "C" rbsc_status rbsc_batch_refine(rbsc_ctx* ctx, const rbsc_csr* graphs, const uint64_t* graph_nodes, uint32_t num_graphs,
                                         const uint32_t* init_colors, rbsc_batch_result* out, rbsc_stats* stats)
{
    if (!ctx) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null context");
    auto t0 = std::chrono::steady_clock::now();
    rbsc_graph* g = nullptr;
    rbsc_status st = rbsc_graph_upload(ctx, graphs, &g);
    if (st != RBSC_OK) return st;
    g->oneshot = true;
    st = rbsc_graph_batch_refine(ctx, g, graph_nodes, num_graphs, init_colors, out, stats);
    rbsc_graph_free(g);
    if (st == RBSC_OK && stats) stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return st;
}
