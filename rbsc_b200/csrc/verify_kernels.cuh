// verify_kernels.cuh -- exact stability check of a hashed fixpoint.
//
// Hash refinement can only merge too much, never split too much: two nodes
// that exact refinement keeps together have equal old colours and equal
// successor-colour multisets, hence equal hashes.  So the hashed fixpoint P is
// coarser than or equal to the coarsest stable partition Q.  If P is also
// stable and refines the initial colouring, P is finer than or equal to Q, and
// P == Q.  This check decides exactly that, without any hashing:
//   for every node u of a non-singleton block with representative r (the
//   block's smallest node): initial colour(u) == initial colour(r), and the
//   multiset {(colour(v), summed weight)} over u's arcs equals r's.
// Short rows (at most 32 arcs, unit weights) are compared in registers: a
// group of 8 or 32 lanes loads u's and r's head colours and bitonic-sorts
// both.  Longer rows and weighted rows go through a global path: their rows
// are turned into keys (row << 31 | head colour), radix-sorted (which sorts
// every row's colours), and u's sorted row is compared with r's.  Nodes that
// fail are split from their block by an exact repair pass, and refinement
// resumes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "refine_kernels.cuh"

namespace rbsc {

struct VerifyLists {
    uint32_t* l8;     // nodes whose row has 1..8 arcs
    uint32_t* l32;    // 9..32 arcs
    uint32_t* llong;  // longer or weighted rows
    uint32_t* counts; // [0] = |l8|, [1] = |l32|, [2] = |llong|, [3] = failures
};

// Classifies every node against its block's representative r (the block's
// smallest node): quick failures (initial colour, row length), empty rows
// (equal), short rows (lists l8 / l32), long or weighted rows (list llong;
// their and r's rows are flagged for the global path in vflag).  Grid-stride
// by warps, 32 consecutive nodes per warp and step, list appends buffered per
// warp (warp_append): a global counter is touched once per ~kWarpBuf listed
// nodes, and no block-wide barrier is needed.  It also writes every node's
// canonical label to `out` (the refinement's result when the check passes,
// so no separate pass over the colours is needed then).
static __global__ void __launch_bounds__(256, 2) k_verify_classify(uint32_t n, const uint32_t* __restrict__ col,
                                                                const uint32_t* __restrict__ initlab,
                                                                const uint64_t* __restrict__ off, int weighted, VerifyLists vl,
                                                                uint32_t* __restrict__ vflag, uint32_t* __restrict__ fail,
                                                                uint32_t* __restrict__ out)
{
    __shared__ uint32_t s_buf[256 / 32][3][kWarpBuf];  // kWarpBuf: common.cuh
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* b8 = s_buf[warp][0];
    uint32_t* b32 = s_buf[warp][1];
    uint32_t* bl = s_buf[warp][2];
    uint32_t c8 = 0, c32 = 0, cl = 0, nbad = 0;
    const uint32_t nwarps = gridDim.x * (256u / 32u);
    // U x 32 consecutive nodes per warp and step: the colour loads of U nodes
    // per lane, then their offset and label loads, are issued side by side,
    // so U dependent chains overlap
    constexpr int U = 4;
    for (uint32_t base = (blockIdx.x * (256u / 32u) + warp) * 32u * U; base < n; base += nwarps * 32u * U) {
        uint32_t c[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + 32u * j + lane;
            c[j] = u < n ? col[u] : kSingleton;
        }
        bool check[U];
        uint64_t ou0[U], ou1[U], or0[U], or1[U];
        uint32_t lu[U], lr[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + 32u * j + lane;
            const uint32_t r = c[j] & kLabelMask;
            if (u < n) out[u] = r;  // the canonical labels, final when the check passes
            check[j] = u < n && !(c[j] & kSingleton) && r != u;
            ou0[j] = ou1[j] = or0[j] = or1[j] = 0ull;
            lu[j] = lr[j] = 0u;
            if (check[j]) {
                ou0[j] = off[u];
                ou1[j] = off[u + 1];
                or0[j] = off[r];
                or1[j] = off[r + 1];
                lu[j] = initlab[u];
                lr[j] = initlab[r];
            }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + 32u * j + lane;
            const uint32_t r = c[j] & kLabelMask;
            bool t8 = false, t32 = false, tl = false, bad = false;
            if (check[j]) {
                const uint64_t du = ou1[j] - ou0[j], dr = or1[j] - or0[j];
                if (lu[j] != lr[j]) bad = true;
                else if (weighted) tl = du > 0 || dr > 0;
                else if (du != dr) bad = true;
                else if (du == 0) {}
                else if (du <= 8) t8 = true;
                else if (du <= 32) t32 = true;
                else tl = true;
                if (tl) {
                    vflag[u] = 1u;
                    vflag[r] = 1u;
                }
                if (bad) fail[u] = 1u;
            }
            warp_append(t8, u, b8, c8, &vl.counts[0], vl.l8);
            warp_append(t32, u, b32, c32, &vl.counts[1], vl.l32);
            warp_append(tl, u, bl, cl, &vl.counts[2], vl.llong);
            nbad += bad ? 1u : 0u;
        }
    }
    warp_append_flush(b8, c8, &vl.counts[0], vl.l8);
    warp_append_flush(b32, c32, &vl.counts[1], vl.l32);
    warp_append_flush(bl, cl, &vl.counts[2], vl.llong);
    nbad = __reduce_add_sync(0xffffffffu, nbad);
    if (lane == 0 && nbad) atomicAdd(&vl.counts[3], nbad);
}

// Bitonic sort of one value per lane across aligned groups of G lanes.
template <int G> __device__ __forceinline__ uint32_t group_sort(uint32_t v)
{
    const int gl = threadIdx.x & (G - 1);
#pragma unroll
    for (int k = 2; k <= G; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (gl & k) == 0;
            const bool lower = (gl & j) == 0;
            v = (lower == up) ? min(v, o) : max(v, o);
        }
    }
    return v;
}

// Groups of G lanes compare the sorted head colours of u and its block's
// representative (rows of equal length <= G, unit weights).
// Rows are read from an arc view: node u's row starts at vstart[u] in idx
// (vstart = off for the graph's own arrays, or the start of u's row in the
// compacted active set, which holds every row the check reads); its length
// is always off[u+1] - off[u].
template <int G>
static __global__ void k_verify_short(uint32_t n, const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                      const uint32_t* __restrict__ col, const uint64_t* __restrict__ off,
                                      const uint64_t* __restrict__ vstart, const uint32_t* __restrict__ idx,
                                      uint32_t* __restrict__ fail, uint32_t* __restrict__ nfail)
{
    const uint32_t cnt = *count;
    const int gl = threadIdx.x & (G - 1);
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    constexpr uint32_t kGroupsPerWarp = 32 / G;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t gw = (threadIdx.x & 31) / G;
    // the loop runs the same number of times on every lane of a warp (the
    // shuffles need all 32); groups past the end carry no work
    for (uint32_t wb = warp * kGroupsPerWarp; wb < cnt; wb += nwarps * kGroupsPerWarp) {
        const uint32_t gi = wb + gw;
        const bool valid = gi < cnt;
        uint32_t a = 0xffffffffu, b = 0xffffffffu;
        uint32_t u = 0;
        if (valid) {
            u = list[gi];
            const uint32_t r = col[u] & kLabelMask;
            const uint64_t ou = vstart[u], orr = vstart[r];
            const uint32_t d = (uint32_t)(off[u + 1] - off[u]);
            if ((uint32_t)gl < d) {
                a = col[idx[ou + gl]] & kLabelMask;
                b = col[idx[orr + gl]] & kLabelMask;
            }
        }
        a = group_sort<G>(a);
        b = group_sort<G>(b);
        const unsigned diff = __ballot_sync(0xffffffffu, a != b) & gmask;
        if (valid && gl == 0 && diff) {
            fail[u] = 1u;
            atomicAdd(nfail, 1u);
        }
    }
}

// vflag[u] = u's row is needed by the global path; vdeg[u] = its length.
static __global__ void k_verify_mark(uint32_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ vflag,
                              uint64_t* __restrict__ vdeg)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    vdeg[u] = vflag[u] ? off[u + 1] - off[u] : 0ull;
}

// Keys of the needed rows: (row index << 31) | colour of the head.
static __global__ void k_verify_keys(uint32_t n, const uint32_t* __restrict__ col, const uint64_t* __restrict__ off,
                              const uint64_t* __restrict__ vstart, const uint32_t* __restrict__ idx,
                              const uint64_t* __restrict__ wt, const uint32_t* __restrict__ vflag,
                              const uint32_t* __restrict__ vrow, const uint64_t* __restrict__ voff,
                              unsigned long long* __restrict__ keys, unsigned long long* __restrict__ vals)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint64_t d = off[u + 1] - off[u];
    if (d == 0 || !vflag[u]) return;
    const uint64_t b = vstart[u];
    const uint64_t row = vrow[u];
    const uint64_t base = voff[u];
    for (uint64_t k = 0; k < d; ++k) {
        keys[base + k] = (row << 31) | (uint64_t)(col[idx[b + k]] & kLabelMask);
        if (vals) vals[base + k] = wt[b + k];
    }
}

// Row starts of the compacted active set's rows (uint32 offsets): the arc
// view of the exact check when the graph's own arcs are in host memory.
static __global__ void k_verify_starts(const ActiveSet* __restrict__ as, uint64_t* __restrict__ vstart)
{
    const uint32_t K = as->K;
    const uint32_t* __restrict__ rows = as->rows;
    const uint32_t* __restrict__ roff = reinterpret_cast<const uint32_t*>(as->roff);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) vstart[rows[k]] = roff[k];
}

// Walks the next run of equal colours in a sorted row segment; returns false
// when the segment is exhausted.  Runs whose weight sum is 0 (mod 2^64) are
// skipped: they are the same as no arc into that block.
__device__ __forceinline__ bool next_run(const unsigned long long* keys, const unsigned long long* vals, uint64_t& i,
                                         uint64_t end, uint32_t& lab, uint64_t& sum)
{
    while (i < end) {
        lab = (uint32_t)(keys[i] & kLabelMask);
        sum = 0;
        while (i < end && (uint32_t)(keys[i] & kLabelMask) == lab) {
            sum += vals ? vals[i] : 1ull;
            ++i;
        }
        if (sum != 0) return true;
    }
    return false;
}

// One warp per node of the long list (grid-stride).  fail[u] = 1 when u's
// row differs from its representative's.
static __global__ void k_verify_compare(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                 const uint32_t* __restrict__ col, const uint32_t* __restrict__ initlab,
                                 const uint64_t* __restrict__ off, const uint64_t* __restrict__ voff,
                                 const unsigned long long* __restrict__ keys, const unsigned long long* __restrict__ vals,
                                 uint32_t* __restrict__ fail, uint32_t* __restrict__ nfail)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint32_t cnt = *count;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < cnt; w += warps) {
        const uint32_t u = list[w];
        const uint32_t c = col[u];
        const uint32_t r = c & kLabelMask;
        if ((c & kSingleton) || r == u) continue;
        bool bad = initlab[u] != initlab[r];
        const uint64_t du = off[u + 1] - off[u], dr = off[r + 1] - off[r];
        if (!bad) {
            if (vals == nullptr) {
                if (du != dr) {
                    bad = true;
                } else if (du > 0) {
                    const unsigned long long* a = keys + voff[u];
                    const unsigned long long* b = keys + voff[r];
                    bool diff = false;
                    for (uint64_t i = lane; i < du && !diff; i += 32)
                        diff = ((a[i] ^ b[i]) & kLabelMask) != 0;
                    bad = __any_sync(0xffffffffu, diff);
                }
            } else if (lane == 0) {
                uint64_t ia = du ? voff[u] : 0, ea = du ? voff[u] + du : 0;
                uint64_t ib = dr ? voff[r] : 0, eb = dr ? voff[r] + dr : 0;
                for (;;) {
                    uint32_t la = 0, lb = 0;
                    uint64_t sa = 0, sb = 0;
                    const bool ha = next_run(keys, vals, ia, ea, la, sa);
                    const bool hb = next_run(keys, vals, ib, eb, lb, sb);
                    if (ha != hb || (ha && (la != lb || sa != sb))) { bad = true; break; }
                    if (!ha) break;
                }
            }
        }
        bad = __shfl_sync(0xffffffffu, bad, 0) || bad;
        if (lane == 0 && bad) {
            fail[u] = 1u;
            atomicAdd(nfail, 1u);
        }
    }
}

}  // namespace rbsc
