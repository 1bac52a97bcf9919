// sortrelabel.cu -- the sort-based relabel (RBSC_RELABEL_SORT).
//
// The reference's relabel (src/rbsc/rbsc.cu:384-396): stable radix sort of the
// nodes by old colour, then by signature, flag every position whose
// (signature, old colour) differs from its predecessor, inclusive-scan the
// flags into dense ids, scatter them back to node order.  Here the same
// lexicographic order is produced by three stable LSD sorts of node ids with
// the hand-written radix sort (keys: the 32-bit second signature, the 64-bit
// signature, the 31-bit old label), and the group of each position gets the
// smallest node id of the group as its label -- the first node of each group,
// because every sort is stable and the node ids start in increasing order.
// The labels are therefore identical to those of the hash-table relabel.
// The sort covers every node (singletons included, as the reference does).
#include <algorithm>
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "radix.cuh"
#include "refine_kernels.cuh"
#include "scan.cuh"

using namespace rbsc;

namespace {

__device__ __forceinline__ uint64_t masked_sig1(const RoundState* st, uint64_t s)
{
    const uint32_t hb = st->hash_bits;
    if (hb) s = (hb >= 64) ? 0ull : (s & ((1ull << hb) - 1ull));
    return s;
}
__device__ __forceinline__ uint32_t masked_sig2(const RoundState* st, uint32_t s) { return st->hash_bits ? 0u : s; }

__global__ void k_sr_init(uint32_t n, const RoundState* __restrict__ st, const Sig* __restrict__ sig,
                          uint32_t* __restrict__ perm, unsigned long long* __restrict__ keys)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        perm[i] = i;
        keys[i] = masked_sig2(st, sig[i].s2);
    }
}

__global__ void k_sr_gather_sig1(uint32_t n, const RoundState* __restrict__ st, const uint32_t* __restrict__ perm,
                                 const Sig* __restrict__ sig, unsigned long long* __restrict__ keys)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = masked_sig1(st, sig[perm[i]].s1);
}

__global__ void k_sr_gather_label(uint32_t n, const uint32_t* __restrict__ col, const uint32_t* __restrict__ perm,
                                  unsigned long long* __restrict__ keys)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = col[perm[i]] & kLabelMask;
}

// head[i] = position i starts a new (label, signature) group
__global__ void k_sr_heads(uint32_t n, const RoundState* __restrict__ st, const uint32_t* __restrict__ col,
                           const uint32_t* __restrict__ perm, const Sig* __restrict__ sig, uint32_t* __restrict__ head)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t h = 1;
    if (i > 0) {
        const uint32_t a = perm[i - 1], b = perm[i];
        h = (col[a] & kLabelMask) != (col[b] & kLabelMask) || masked_sig1(st, sig[a].s1) != masked_sig1(st, sig[b].s1) ||
            masked_sig2(st, sig[a].s2) != masked_sig2(st, sig[b].s2);
    }
    head[i] = h;
}

__global__ void k_sr_gstart(uint32_t n, const uint32_t* __restrict__ head, const uint32_t* __restrict__ gid,
                            uint32_t* __restrict__ gstart)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && head[i]) gstart[gid[i]] = i;
}

// New colours in place (the sorts and group flags were computed from the old
// ones in the previous kernels); also zeroes the signatures of the rows that
// cross a tile edge of the current arc set.
__global__ void k_sr_assign(uint32_t n, const ActiveSet* __restrict__ as, uint32_t* __restrict__ col,
                            const uint32_t* __restrict__ perm, const uint32_t* __restrict__ head,
                            const uint32_t* __restrict__ gid, const uint32_t* __restrict__ gstart,
                            Sig* __restrict__ sig)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t grp = head[i] ? gid[i] : gid[i] - 1u;
        const bool single = head[i] && (i + 1 == n || head[i + 1]);
        col[perm[i]] = perm[gstart[grp]] | (single ? kSingleton : 0u);
    }
    const uint32_t nsplit = as->nsplit;
    const uint32_t* __restrict__ split_rows = as->split;
    for (uint32_t k = i; k < nsplit; k += gridDim.x * blockDim.x) {
        const uint32_t node = split_rows[k];
        sig_store(&sig[node], 0ull, 0u);
    }
}

}  // namespace

void sortrelabel_release(rbsc_graph* g)
{
    dev_free(g->ctx, (void*&)g->d_sr_keys[0]);
    dev_free(g->ctx, (void*&)g->d_sr_keys[1]);
    dev_free(g->ctx, (void*&)g->d_sr_perm[0]);
    dev_free(g->ctx, (void*&)g->d_sr_perm[1]);
    dev_free(g->ctx, (void*&)g->d_sr_head);
    dev_free(g->ctx, (void*&)g->d_sr_gstart);
    dev_free(g->ctx, g->d_sr_tmp);
    g->sr_tmp_bytes = 0;
    g->sr_bufs = false;
}

rbsc_status ensure_sort_relabel_bufs(rbsc_ctx* ctx, rbsc_graph* g)
{
    if (ctx->opts.relabel != RBSC_RELABEL_SORT || g->sr_bufs) return RBSC_OK;
    const size_t n = std::max<uint32_t>(g->n, 1);
    rbsc_status st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_keys[0], 8 * n)) != RBSC_OK) return st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_keys[1], 8 * n)) != RBSC_OK) return st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_perm[0], 4 * n)) != RBSC_OK) return st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_perm[1], 4 * n)) != RBSC_OK) return st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_head, 4 * (n + 1))) != RBSC_OK) return st;
    if ((st = dev_alloc(ctx, (void**)&g->d_sr_gstart, 4 * n)) != RBSC_OK) return st;
    g->sr_tmp_bytes = std::max(radix_temp_bytes(n), scan_temp_bytes<uint32_t>(n)) + 1024;
    if ((st = dev_alloc(ctx, &g->d_sr_tmp, g->sr_tmp_bytes)) != RBSC_OK) return st;
    g->sr_bufs = true;
    return RBSC_OK;
}

// Launches one sort-based relabel on stream s (capturable: no host syncs).
rbsc_status launch_sort_relabel(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s)
{
    const uint32_t n = g->n;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, ceil_div<uint64_t>(n, 256));
    unsigned long long *k0 = g->d_sr_keys[0], *k1 = g->d_sr_keys[1];
    uint32_t *p0 = g->d_sr_perm[0], *p1 = g->d_sr_perm[1];
    bool alt = false;
    cudaError_t e;
    ++rbsc::launch_counter();
    k_sr_init<<<grid, 256, 0, s>>>(n, g->d_st, g->d_sig, p0, k0);
    if ((e = radix_sort<uint32_t>(k0, k1, p0, p1, n, 0, 32, g->d_sr_tmp, s, &alt)) != cudaSuccess)
        return rbsc_cuda_fail(ctx, e, "radix_sort (sig2)", __LINE__);
    if (alt) { std::swap(k0, k1); std::swap(p0, p1); }
    ++rbsc::launch_counter();
    k_sr_gather_sig1<<<grid, 256, 0, s>>>(n, g->d_st, p0, g->d_sig, k0);
    if ((e = radix_sort<uint32_t>(k0, k1, p0, p1, n, 0, 64, g->d_sr_tmp, s, &alt)) != cudaSuccess)
        return rbsc_cuda_fail(ctx, e, "radix_sort (sig1)", __LINE__);
    if (alt) { std::swap(k0, k1); std::swap(p0, p1); }
    ++rbsc::launch_counter();
    k_sr_gather_label<<<grid, 256, 0, s>>>(n, g->d_col[0], p0, k0);
    if ((e = radix_sort<uint32_t>(k0, k1, p0, p1, n, 0, 31, g->d_sr_tmp, s, &alt)) != cudaSuccess)
        return rbsc_cuda_fail(ctx, e, "radix_sort (label)", __LINE__);
    if (alt) { std::swap(k0, k1); std::swap(p0, p1); }
    // p0 = sorted node order; p1 is free: use it for the group ids
    ++rbsc::launch_counter();
    k_sr_heads<<<grid, 256, 0, s>>>(n, g->d_st, g->d_col[0], p0, g->d_sig, g->d_sr_head);
    uint32_t* count = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(g->d_st) + offsetof(RoundState, count));
    if ((e = exclusive_scan<uint32_t, uint32_t>(g->d_sr_head, p1, n, count, g->d_sr_tmp, s)) != cudaSuccess)
        return rbsc_cuda_fail(ctx, e, "exclusive_scan (heads)", __LINE__);
    ++rbsc::launch_counter();
    k_sr_gstart<<<grid, 256, 0, s>>>(n, g->d_sr_head, p1, g->d_sr_gstart);
    ++rbsc::launch_counter();
    k_sr_assign<<<grid, 256, 0, s>>>(n, g->d_as, g->d_col[0], p0, g->d_sr_head, p1, g->d_sr_gstart, g->d_sig);
    if ((e = cudaGetLastError()) != cudaSuccess) return rbsc_cuda_fail(ctx, e, "sort relabel launch", __LINE__);
    return RBSC_OK;
}
