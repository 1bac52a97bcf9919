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
// The rows of all nodes in non-singleton blocks are turned into keys
// (row << 31 | head colour), radix-sorted (which sorts every row's colours),
// and u's sorted row is compared with r's.  Nodes that fail are split from
// their block by an exact repair pass, and refinement resumes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace rbsc {

// vflag[u] = u's row is needed by the check; vdeg[u] = its length if needed.
static __global__ void k_verify_mark(uint32_t n, const uint32_t* __restrict__ col, const uint64_t* __restrict__ off,
                              uint32_t* __restrict__ vflag, uint64_t* __restrict__ vdeg)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint64_t d = off[u + 1] - off[u];
    const bool need = !(col[u] & kSingleton) && d > 0;
    vflag[u] = need ? 1u : 0u;
    vdeg[u] = need ? d : 0ull;
}

// Keys of the needed rows: (row index << 31) | colour of the head.
static __global__ void k_verify_keys(uint32_t n, const uint32_t* __restrict__ col, const uint64_t* __restrict__ off,
                              const uint32_t* __restrict__ idx, const uint64_t* __restrict__ wt,
                              const uint32_t* __restrict__ vrow, const uint64_t* __restrict__ voff,
                              unsigned long long* __restrict__ keys, unsigned long long* __restrict__ vals)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint64_t b = off[u], e = off[u + 1];
    if (e == b || (col[u] & kSingleton)) return;
    const uint64_t row = vrow[u];
    const uint64_t base = voff[u];
    for (uint64_t k = b; k < e; ++k) {
        keys[base + (k - b)] = (row << 31) | (uint64_t)(col[idx[k]] & kLabelMask);
        if (vals) vals[base + (k - b)] = wt[k];
    }
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

// One warp per node (grid-stride).  fail[u] = 1 when u's row differs from its
// representative's.
static __global__ void k_verify_compare(uint32_t n, const uint32_t* __restrict__ col, const uint32_t* __restrict__ initlab,
                                 const uint64_t* __restrict__ off, const uint64_t* __restrict__ voff,
                                 const unsigned long long* __restrict__ keys, const unsigned long long* __restrict__ vals,
                                 uint32_t* __restrict__ fail, uint32_t* __restrict__ nfail)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
        const uint32_t u = (uint32_t)w;
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
