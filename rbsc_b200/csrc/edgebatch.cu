// edgebatch.cu -- the reference's edge-batch (quotient) mode on the device.
//
// src/rbsc/rbsc.cu:292-487 refines a graph whose arcs do not fit one batch
// in an outer loop.  Each iteration cuts the arc list (grouped by start) into
// batches of edge_batch_size arcs, trims every batch to the runs of arcs that
// start and end inside it, and refines each batch on its own: its sources
// start in one block, nodes without any arc (batch 0 only) in another, every
// other node alone.  The classes of a batch get fresh global ids in the order
// of their smallest node; nodes in no batch get ids of their own.  The graph
// is then replaced by its quotient: the first run of every class (in arc
// order) is kept, heads are renamed to classes and parallel arcs merged with
// their weights summed.  The loop ends when an iteration had one batch (the
// result is then the coarsest partition: done = 1) or the node count did not
// shrink (done = 0); rbsc_aggressive.cu:487 also stops when the batch count
// would not shrink.
//
// Here the arc list lives on the device in "run form": runs k = 0..R-1 with
// source rsrc[k] and arcs [roff[k], roff[k+1]) of heads dst and weights wt,
// runs in the reference's arc order.  Every batch is refined with this
// library's exact refinement (the reference hashes; the partitions agree
// unless its 64-bit sums collide), its local graph built on the device as a
// CSR over all nodes.  The quotient keeps the runs' order; inside a run the
// merged arcs come out sorted by head class, which changes no later result
// (a run's arcs are summed, in any order).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "common.cuh"
#include "radix.cuh"
#include "scan.cuh"
#include "internal.h"

using namespace rbsc;

namespace {

constexpr uint32_t kNone = 0xffffffffu;

unsigned grid_of(uint64_t n, unsigned t = 256)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + t - 1) / t, 65535ull * 64));
}

// run form of a CSR: one run per non-empty row, in node order
__global__ void k_eb_row_flags(uint32_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ flag)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        flag[u] = off[u + 1] > off[u] ? 1u : 0u;
}

__global__ void k_eb_runs_from_rows(uint32_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ pos,
                                    uint32_t* __restrict__ rsrc, uint64_t* __restrict__ roff)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        if (off[u + 1] > off[u]) {
            rsrc[pos[u]] = (uint32_t)u;
            roff[pos[u]] = off[u];
        }
}

// has[v] = 1 for every node that starts a run
__global__ void k_eb_has_run(uint32_t R, const uint32_t* __restrict__ rsrc, uint8_t* __restrict__ has)
{
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < R; k += (uint64_t)gridDim.x * blockDim.x)
        has[rsrc[k]] = 1;
}

// local CSR of runs [k0, k1): row lengths, then the arcs (one warp per run)
__global__ void k_eb_local_deg(uint32_t k0, uint32_t k1, const uint32_t* __restrict__ rsrc, const uint64_t* __restrict__ roff,
                               uint64_t* __restrict__ deg)
{
    for (uint64_t k = k0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < k1; k += (uint64_t)gridDim.x * blockDim.x)
        deg[rsrc[k]] = roff[k + 1] - roff[k];
}

__global__ void k_eb_local_fill(uint32_t k0, uint32_t k1, const uint32_t* __restrict__ rsrc, const uint64_t* __restrict__ roff,
                                const uint32_t* __restrict__ dst, const uint64_t* __restrict__ wt,
                                const uint64_t* __restrict__ loff, uint32_t* __restrict__ lidx, uint64_t* __restrict__ lwt)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = k0 + ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5); k < k1; k += warps) {
        const uint64_t a = roff[k], len = roff[k + 1] - a, o = loff[rsrc[k]];
        for (uint64_t j = lane; j < len; j += 32) {
            lidx[o + j] = dst[a + j];
            if (lwt) lwt[o + j] = wt[a + j];
        }
    }
}

// initial colours of a batch: sources 0, arc-less nodes 1 (batch 0), others alone
__global__ void k_eb_local_init(uint32_t n, const uint8_t* __restrict__ has, int first_batch, uint32_t* __restrict__ col)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        col[u] = (first_batch && !has[u]) ? 1u : (uint32_t)u + 2u;
}

__global__ void k_eb_mark_sources(uint32_t k0, uint32_t k1, const uint32_t* __restrict__ rsrc, uint32_t* __restrict__ col)
{
    for (uint64_t k = k0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < k1; k += (uint64_t)gridDim.x * blockDim.x)
        col[rsrc[k]] = 0u;
}

// members of the batch (colour 0 or 1) that carry their block's label
__global__ void k_eb_rep_flags(uint32_t n, const uint32_t* __restrict__ lab, const uint32_t* __restrict__ col,
                               uint32_t* __restrict__ flag)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        flag[u] = (col[u] <= 1u && lab[u] == (uint32_t)u) ? 1u : 0u;
}

__global__ void k_eb_assign(uint32_t n, const uint32_t* __restrict__ lab, const uint32_t* __restrict__ col,
                            const uint32_t* __restrict__ rank, uint32_t base, uint32_t* __restrict__ w)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        if (col[u] <= 1u) w[u] = base + rank[lab[u]];
}

__global__ void k_eb_unassigned_flags(uint32_t n, const uint32_t* __restrict__ w, uint32_t* __restrict__ flag)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        flag[u] = w[u] == kNone ? 1u : 0u;
}

__global__ void k_eb_assign_rest(uint32_t n, const uint32_t* __restrict__ rank, uint32_t base, uint32_t* __restrict__ w)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        if (w[u] == kNone) w[u] = base + rank[u];
}

__global__ void k_eb_iota(uint32_t n, uint32_t* __restrict__ out)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        out[u] = (uint32_t)u;
}

__global__ void k_eb_compose(uint32_t n, const uint32_t* __restrict__ w, uint32_t* __restrict__ cls)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        cls[u] = w[cls[u]];
}

// quotient: the first run (in arc order) of every class is kept
__global__ void k_eb_first_run(uint32_t R, const uint32_t* __restrict__ rsrc, const uint32_t* __restrict__ w,
                               uint32_t* __restrict__ first)
{
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < R; k += (uint64_t)gridDim.x * blockDim.x)
        atomicMin(&first[w[rsrc[k]]], (uint32_t)k);
}

__global__ void k_eb_keep(uint32_t R, const uint32_t* __restrict__ rsrc, const uint32_t* __restrict__ w,
                          const uint32_t* __restrict__ first, const uint64_t* __restrict__ roff, uint32_t* __restrict__ keep,
                          uint64_t* __restrict__ klen)
{
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < R; k += (uint64_t)gridDim.x * blockDim.x) {
        const bool kp = first[w[rsrc[k]]] == (uint32_t)k;
        keep[k] = kp ? 1u : 0u;
        klen[k] = kp ? roff[k + 1] - roff[k] : 0ull;
    }
}

// keys (kept run rank << 32 | head class), values weights; one warp per run
__global__ void k_eb_keys(uint32_t R, const uint64_t* __restrict__ roff, const uint32_t* __restrict__ dst,
                          const uint64_t* __restrict__ wt, const uint32_t* __restrict__ w, const uint32_t* __restrict__ keep,
                          const uint32_t* __restrict__ krank, const uint64_t* __restrict__ kpos,
                          unsigned long long* __restrict__ keys, unsigned long long* __restrict__ vals)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; k < R; k += warps) {
        if (!keep[k]) continue;
        const uint64_t a = roff[k], len = roff[k + 1] - a, o = kpos[k];
        const unsigned long long hi = (unsigned long long)krank[k] << 32;
        for (uint64_t j = lane; j < len; j += 32) {
            keys[o + j] = hi | w[dst[a + j]];
            vals[o + j] = wt ? wt[a + j] : 1ull;
        }
    }
}

__global__ void k_eb_heads(uint64_t n, const unsigned long long* __restrict__ keys, uint32_t* __restrict__ head)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// one merged arc per segment of equal keys; a new run where the run rank changes
__global__ void k_eb_merge(uint64_t n, const unsigned long long* __restrict__ keys, const unsigned long long* __restrict__ vals,
                           const uint32_t* __restrict__ head, const uint64_t* __restrict__ hpos, uint32_t* __restrict__ ndst,
                           uint64_t* __restrict__ nwt, uint64_t* __restrict__ nroff)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        const unsigned long long k = keys[i];
        unsigned long long s = vals[i];
        for (uint64_t j = i + 1; j < n && keys[j] == k; ++j) s += vals[j];
        const uint64_t p = hpos[i];
        ndst[p] = (uint32_t)k;
        nwt[p] = s;
        if (i == 0 || (keys[i - 1] >> 32) != (k >> 32)) nroff[k >> 32] = p;
    }
}

__global__ void k_eb_new_src(uint32_t R, const uint32_t* __restrict__ rsrc, const uint32_t* __restrict__ w,
                             const uint32_t* __restrict__ keep, const uint32_t* __restrict__ krank, uint32_t* __restrict__ nrsrc)
{
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < R; k += (uint64_t)gridDim.x * blockDim.x)
        if (keep[k]) nrsrc[krank[k]] = w[rsrc[k]];
}

// canonical labels of the original nodes: smallest node of each final class
__global__ void k_eb_min_node(uint32_t n, const uint32_t* __restrict__ cls, uint32_t* __restrict__ first)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        atomicMin(&first[cls[u]], (uint32_t)u);
}

__global__ void k_eb_labels(uint32_t n, const uint32_t* __restrict__ cls, const uint32_t* __restrict__ first,
                            uint32_t* __restrict__ out)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        out[u] = first[cls[u]];
}

// The arc list in run form, with its buffers (device).
struct Runs {
    uint32_t R = 0;
    uint64_t E = 0;
    uint32_t* rsrc = nullptr;
    uint64_t* roff = nullptr;
    uint32_t* dst = nullptr;
    uint64_t* wt = nullptr;  // null: every weight 1
};

// The local graph of runs [k0, k1) over n nodes, refined exactly from the
// batch's initial colours; canonical labels into lab.
rbsc_status refine_batch(rbsc_ctx* ctx, const Runs& rs, uint32_t n, uint32_t k0, uint32_t k1, const uint8_t* has, bool first_batch,
                         uint32_t* col, uint32_t* lab, uint32_t* rounds)
{
    cudaStream_t s = ctx->stream;
    uint64_t a0 = 0, a1 = 0;
    EK(cudaMemcpyAsync(&a0, rs.roff + k0, 8, cudaMemcpyDeviceToHost, s));
    EK(cudaMemcpyAsync(&a1, rs.roff + k1, 8, cudaMemcpyDeviceToHost, s));
    EK(cudaStreamSynchronize(s));
    rbsc_graph* g = new (std::nothrow) rbsc_graph();
    if (!g) return rbsc_fail(ctx, RBSC_ERR_OOM, "out of host memory");
    struct Free { rbsc_graph* g; ~Free() { rbsc_graph_free(g); } } guard{g};
    g->ctx = ctx;
    g->n = n;
    g->m = a1 - a0;
    g->oneshot = true;
    EKS(graph_alloc_csr(ctx, g, rs.wt != nullptr));
    EK(cudaMemsetAsync(g->d_off, 0, 8 * ((size_t)n + 1), s));
    ++rbsc::launch_counter();
    k_eb_local_deg<<<grid_of(k1 - k0), 256, 0, s>>>(k0, k1, rs.rsrc, rs.roff, g->d_off);
    EK(cudaGetLastError());
    void* tmp = nullptr;
    EKS(dev_alloc(ctx, &tmp, scan_temp_bytes<uint64_t>((uint64_t)n + 1) + 1024));
    struct FreeTmp { rbsc_ctx* c; void*& p; ~FreeTmp() { dev_free(c, p); } } guard2{ctx, tmp};
    EK((exclusive_scan<uint64_t, uint64_t>(g->d_off, g->d_off, n, g->d_off + n, tmp, s)));
    ++rbsc::launch_counter();
    k_eb_local_fill<<<grid_of((uint64_t)(k1 - k0) * 32), 256, 0, s>>>(k0, k1, rs.rsrc, rs.roff, rs.dst, rs.wt, g->d_off, g->d_idx,
                                                                    g->d_wt);
    ++rbsc::launch_counter();
    k_eb_local_init<<<grid_of(n), 256, 0, s>>>(n, has, first_batch ? 1 : 0, col);
    ++rbsc::launch_counter();
    k_eb_mark_sources<<<grid_of(k1 - k0), 256, 0, s>>>(k0, k1, rs.rsrc, col);
    EK(cudaGetLastError());
    EKS(graph_prepare(ctx, g));
    rbsc_stats st;
    EKS(refine_resident(ctx, g, col, lab, &st, nullptr));
    *rounds += st.rounds;
    return RBSC_OK;
}

}  // namespace

extern "C" rbsc_status rbsc_refine_edge_batches(rbsc_ctx* ctx, const rbsc_csr* host_graph, uint64_t edge_batch_size,
                                                int32_t aggressive, uint32_t* out_labels, rbsc_stats* stats,
                                                rbsc_edge_batch_info* info)
{
    if (!ctx) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null context");
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof *stats);
    if (info) std::memset(info, 0, sizeof *info);
    const uint64_t lc0 = rbsc::launch_counter();
    // upload (validates the CSR) and the run form of its rows
    rbsc_graph* in = nullptr;
    EKS(rbsc_graph_upload(ctx, host_graph, &in));
    struct FreeIn { rbsc_graph*& g; ~FreeIn() { rbsc_graph_free(g); } } guard_in{in};
    cudaStream_t s = ctx->stream;
    const uint32_t N = in->n;
    const uint64_t E = in->m;
    const uint64_t B = edge_batch_size ? edge_batch_size : std::max<uint64_t>(E, 1);
    Scratch sc(ctx);
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    auto need_tmp = [&](size_t bytes) -> rbsc_status {
        if (bytes <= tmp_bytes) return RBSC_OK;
        if (tmp) sc.release(tmp);
        tmp_bytes = 0;
        rbsc_status st = sc.get((char**)&tmp, bytes);
        if (st == RBSC_OK) tmp_bytes = bytes;
        return st;
    };
    Runs cur, nxt;
    uint32_t *cls = nullptr, *w = nullptr, *col = nullptr, *lab = nullptr, *flag = nullptr, *small = nullptr;
    uint8_t* has = nullptr;
    EKS(sc.get(&cls, N));
    EKS(sc.get(&w, N));
    EKS(sc.get(&col, N));
    EKS(sc.get(&lab, N));
    EKS(sc.get(&flag, (size_t)N + 1));
    EKS(sc.get(&has, N));
    EKS(sc.get(&small, 16));
    EKS(sc.get(&cur.rsrc, N));
    EKS(sc.get(&cur.roff, (size_t)N + 1));
    EKS(sc.get(&cur.dst, E));
    if (in->weighted) EKS(sc.get(&cur.wt, E));
    {
        // identity classes, runs = non-empty rows
        EKS(need_tmp(scan_temp_bytes<uint32_t>((uint64_t)N + 1) + 1024));
        ++rbsc::launch_counter();
        k_eb_row_flags<<<grid_of(N), 256, 0, s>>>(N, in->d_off, flag);
        EK((exclusive_scan<uint32_t, uint32_t>(flag, flag, N, small, tmp, s)));
        ++rbsc::launch_counter();
        k_eb_runs_from_rows<<<grid_of(N), 256, 0, s>>>(N, in->d_off, flag, cur.rsrc, cur.roff);
        EK(cudaGetLastError());
        EK(cudaMemcpyAsync(&cur.R, small, 4, cudaMemcpyDeviceToHost, s));
        if (E) EK(cudaMemcpyAsync(cur.dst, in->d_idx, 4 * E, cudaMemcpyDeviceToDevice, s));
        if (cur.wt && E) EK(cudaMemcpyAsync(cur.wt, in->d_wt, 8 * E, cudaMemcpyDeviceToDevice, s));
        EK(cudaStreamSynchronize(s));
        cur.E = E;
        EK(cudaMemcpyAsync(cur.roff + cur.R, &cur.E, 8, cudaMemcpyHostToDevice, s));
        ++rbsc::launch_counter();
        k_eb_iota<<<grid_of(N), 256, 0, s>>>(N, cls);
        EK(cudaGetLastError());
        EK(cudaStreamSynchronize(s));
    }
    rbsc_graph_free(in);
    in = nullptr;

    uint32_t node_n = N, new_node_n = N, iters = 0, rounds = 0;
    uint64_t batches = 0, batches_total = 0, refinements = 0;
    std::vector<uint64_t> roff_h;
    for (;;) {
        node_n = new_node_n;
        new_node_n = 0;
        const uint64_t edge_n = cur.E;
        batches = (uint64_t)std::ceil((double)edge_n / (double)B);
        batches_total += batches;
        EK(cudaMemsetAsync(w, 0xff, 4 * (size_t)std::max<uint32_t>(node_n, 1), s));
        EK(cudaMemsetAsync(has, 0, std::max<uint32_t>(node_n, 1), s));
        ++rbsc::launch_counter();
        k_eb_has_run<<<grid_of(cur.R), 256, 0, s>>>(cur.R, cur.rsrc, has);
        EK(cudaGetLastError());
        roff_h.resize((size_t)cur.R + 1);
        EK(cudaMemcpyAsync(roff_h.data(), cur.roff, 8 * ((size_t)cur.R + 1), cudaMemcpyDeviceToHost, s));
        EK(cudaStreamSynchronize(s));
        EKS(need_tmp(scan_temp_bytes<uint32_t>((uint64_t)node_n + 1) + 1024));
        for (uint64_t b = 0; b < batches; ++b) {
            // trimmed to the runs that start at or after bs and end at or before be
            const uint64_t bs = b * B, be = std::min(edge_n, bs + B);
            const uint32_t k0 = (uint32_t)(std::lower_bound(roff_h.begin(), roff_h.end() - 1, bs) - roff_h.begin());
            if (k0 >= cur.R || roff_h[k0] >= be) continue;
            const uint32_t k1 = (uint32_t)(std::upper_bound(roff_h.begin() + k0, roff_h.end(), be) - roff_h.begin()) - 1;
            if (k1 <= k0) continue;
            EKS(refine_batch(ctx, cur, node_n, k0, k1, has, b == 0, col, lab, &rounds));
            ++refinements;
            // fresh ids for the batch's classes, in the order of their smallest node
            ++rbsc::launch_counter();
            k_eb_rep_flags<<<grid_of(node_n), 256, 0, s>>>(node_n, lab, col, flag);
            EK((exclusive_scan<uint32_t, uint32_t>(flag, flag, node_n, small, tmp, s)));
            ++rbsc::launch_counter();
            k_eb_assign<<<grid_of(node_n), 256, 0, s>>>(node_n, lab, col, flag, new_node_n, w);
            EK(cudaGetLastError());
            uint32_t added = 0;
            EK(cudaMemcpyAsync(&added, small, 4, cudaMemcpyDeviceToHost, s));
            EK(cudaStreamSynchronize(s));
            new_node_n += added;
        }
        ++iters;
        if (batches > 1) {
            // nodes in no batch: ids of their own, in node order
            ++rbsc::launch_counter();
            k_eb_unassigned_flags<<<grid_of(node_n), 256, 0, s>>>(node_n, w, flag);
            EK((exclusive_scan<uint32_t, uint32_t>(flag, flag, node_n, small, tmp, s)));
            ++rbsc::launch_counter();
            k_eb_assign_rest<<<grid_of(node_n), 256, 0, s>>>(node_n, flag, new_node_n, w);
            EK(cudaGetLastError());
            uint32_t added = 0;
            EK(cudaMemcpyAsync(&added, small, 4, cudaMemcpyDeviceToHost, s));
            EK(cudaStreamSynchronize(s));
            new_node_n += added;
        }
        if (batches > 0) {
            ++rbsc::launch_counter();
            k_eb_compose<<<grid_of(N), 256, 0, s>>>(N, w, cls);
            EK(cudaGetLastError());
        }
        if (!(batches > 1 && node_n > new_node_n)) break;
        // quotient: the first run of every class, heads renamed, parallel arcs merged
        uint32_t *first = nullptr, *keep = nullptr, *krank = nullptr, *head = nullptr;
        uint64_t *klen = nullptr, *hpos = nullptr;
        unsigned long long *keys = nullptr, *keys2 = nullptr, *vals = nullptr, *vals2 = nullptr;
        Scratch q(ctx);
        EKS(q.get(&first, new_node_n));
        EKS(q.get(&keep, cur.R));
        EKS(q.get(&krank, (size_t)cur.R + 1));
        EKS(q.get(&klen, (size_t)cur.R + 1));
        EK(cudaMemsetAsync(first, 0xff, 4 * (size_t)std::max<uint32_t>(new_node_n, 1), s));
        ++rbsc::launch_counter();
        k_eb_first_run<<<grid_of(cur.R), 256, 0, s>>>(cur.R, cur.rsrc, w, first);
        ++rbsc::launch_counter();
        k_eb_keep<<<grid_of(cur.R), 256, 0, s>>>(cur.R, cur.rsrc, w, first, cur.roff, keep, klen);
        EK(cudaGetLastError());
        EKS(need_tmp(std::max(scan_temp_bytes<uint32_t>((uint64_t)cur.R + 1), scan_temp_bytes<uint64_t>((uint64_t)cur.R + 1)) + 1024));
        EK((exclusive_scan<uint32_t, uint32_t>(keep, krank, cur.R, krank + cur.R, tmp, s)));
        EK((exclusive_scan<uint64_t, uint64_t>(klen, klen, cur.R, klen + cur.R, tmp, s)));
        uint32_t R2 = 0;
        uint64_t E2 = 0;
        EK(cudaMemcpyAsync(&R2, krank + cur.R, 4, cudaMemcpyDeviceToHost, s));
        EK(cudaMemcpyAsync(&E2, klen + cur.R, 8, cudaMemcpyDeviceToHost, s));
        EK(cudaStreamSynchronize(s));
        EKS(q.get(&keys, E2));
        EKS(q.get(&keys2, E2));
        EKS(q.get(&vals, E2));
        EKS(q.get(&vals2, E2));
        ++rbsc::launch_counter();
        k_eb_keys<<<grid_of((uint64_t)cur.R * 32), 256, 0, s>>>(cur.R, cur.roff, cur.dst, cur.wt, w, keep, krank, klen, keys, vals);
        EK(cudaGetLastError());
        int rbits = 0;
        while (rbits < 32 && (1ull << rbits) < (uint64_t)R2) ++rbits;
        EKS(need_tmp(std::max(radix_temp_bytes(E2), scan_temp_bytes<uint64_t>(E2 + 1)) + 1024));
        bool alt = false;
        EK(radix_sort<unsigned long long>(keys, keys2, vals, vals2, E2, 0, 32 + rbits, tmp, s, &alt));
        if (alt) {
            std::swap(keys, keys2);
            std::swap(vals, vals2);
        }
        EKS(q.get(&head, E2));
        EKS(q.get(&hpos, E2 + 1));
        ++rbsc::launch_counter();
        k_eb_heads<<<grid_of(E2), 256, 0, s>>>(E2, keys, head);
        EK(cudaGetLastError());
        EK((exclusive_scan<uint32_t, uint64_t>(head, hpos, E2, hpos + E2, tmp, s)));
        uint64_t E3 = 0;
        EK(cudaMemcpyAsync(&E3, hpos + E2, 8, cudaMemcpyDeviceToHost, s));
        EK(cudaStreamSynchronize(s));
        // the next run form (its buffers replace the current ones)
        Runs nr;
        nr.R = R2;
        nr.E = E3;
        EKS(sc.get(&nr.rsrc, R2));
        EKS(sc.get(&nr.roff, (size_t)R2 + 1));
        EKS(sc.get(&nr.dst, E3));
        EKS(sc.get(&nr.wt, E3));
        ++rbsc::launch_counter();
        k_eb_merge<<<grid_of(E2), 256, 0, s>>>(E2, keys, vals, head, hpos, nr.dst, nr.wt, nr.roff);
        ++rbsc::launch_counter();
        k_eb_new_src<<<grid_of(cur.R), 256, 0, s>>>(cur.R, cur.rsrc, w, keep, krank, nr.rsrc);
        EK(cudaGetLastError());
        EK(cudaMemcpyAsync(nr.roff + R2, &nr.E, 8, cudaMemcpyHostToDevice, s));
        EK(cudaStreamSynchronize(s));
        sc.release(cur.rsrc);
        sc.release(cur.roff);
        sc.release(cur.dst);
        if (cur.wt) sc.release(cur.wt);
        cur = nr;
        if (aggressive) {
            // rbsc_aggressive.cu:487: also stop when the batch count would not shrink
            const float next = std::ceil((float)cur.E / (float)B);
            if (!((float)batches > next)) break;
        }
    }
    // canonical labels of the original nodes
    if (out_labels && N) {
        uint32_t* firstn = nullptr;
        if (batches == 0) {
            // no arc at all: one block
            EK(cudaMemsetAsync(cls, 0, 4 * (size_t)N, s));
        }
        EKS(sc.get(&firstn, std::max<uint32_t>(new_node_n, 1)));
        EK(cudaMemsetAsync(firstn, 0xff, 4 * (size_t)std::max<uint32_t>(new_node_n, 1), s));
        ++rbsc::launch_counter();
        k_eb_min_node<<<grid_of(N), 256, 0, s>>>(N, cls, firstn);
        ++rbsc::launch_counter();
        k_eb_labels<<<grid_of(N), 256, 0, s>>>(N, cls, firstn, lab);
        EK(cudaGetLastError());
        EK(cudaMemcpyAsync(out_labels, lab, 4 * (size_t)N, cudaMemcpyDeviceToHost, s));
    }
    EK(cudaStreamSynchronize(s));
    if (stats) {
        stats->blocks = new_node_n;
        stats->done = batches == 1 ? 1u : 0u;
        stats->rounds = rounds;
        stats->verified = 1;
        stats->kernel_launches = rbsc::launch_counter() - lc0;
        stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (info) {
        info->iterations = iters;
        info->last_batches = (uint32_t)std::min<uint64_t>(batches, 0xffffffffu);
        info->batches_total = batches_total;
        info->local_refinements = refinements;
        info->last_arcs = cur.E;
    }
    return RBSC_OK;
}
