// Hot heads of the first signature pass.
//
// The first pass of a refinement with at most 256 initial classes gathers a
// 1-byte class rank per arc.  The gather of scattered bytes is bound by the
// L1's tag stage (about one scattered sector per SM and cycle: R-MAT-24's
// 263 M arcs over 148 SMs take ~0.9 ms), not by HBM.  Shared memory serves a
// warp's 32 scattered bytes in a few cycles, and on graphs with skewed
// in-degrees a small set of nodes receives a large share of the arcs
// (R-MAT-24: the 2^17 most pointed-to nodes receive 56 % of them).  So, once
// per resident graph:
//   * count the in-arcs of every node (k_hot_indeg), pick a threshold from a
//     log-linear histogram (k_hot_hist) so that at most H nodes reach it, and
//     number those nodes in id order (the hot slots; k_hot_flags, a scan,
//     k_hot_assign);
//   * write a second copy of the heads in which a hot head v is replaced by
//     kHotFlag | slot(v) (k_hot_encode).
// Per refinement: hot_rank[slot] = rank[hot_node[slot]] (k_hot_ranks), and
// k_signature_hot stages hot_rank in shared memory, then folds the tiles like
// k_signature, gathering s_hot[slot] for a hot head and rank[v] otherwise.
// The later passes read the plain heads; the result does not depend on
// which nodes are hot.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "refine_kernels.cuh"

namespace rbsc {

constexpr int kHotThreads = 1024;      // one block per SM: 32 warps, the table once per SM
constexpr uint32_t kHotBins = 928;     // log-linear in-degree bins (hot_bin)
constexpr uint32_t kHotMaxLog2 = 17;   // 128 KB of 1-byte ranks in shared memory
constexpr uint32_t kHotMinLog2 = 10;

// Bin of an in-degree: exact below 128, then 32 bins per octave (bins
// 3 % wide, so the threshold admits close to the limit).
__host__ __device__ __forceinline__ uint32_t hot_bin(uint32_t d)
{
    if (d < 128u) return d;
#ifdef __CUDA_ARCH__
    const uint32_t lg = 31u - (uint32_t)__clz(d);
#else
    const uint32_t lg = 31u - (uint32_t)__builtin_clz(d);
#endif
    return 128u + 32u * (lg - 7u) + ((d >> (lg - 5u)) & 31u);
}

// Smallest in-degree of bin b.
__host__ __device__ __forceinline__ uint32_t hot_bin_floor(uint32_t b)
{
    if (b < 128u) return b;
    const uint32_t lg = 7u + (b - 128u) / 32u;
    return (32u + (b - 128u) % 32u) << (lg - 5u);
}

static __global__ void k_hot_indeg(const uint32_t* __restrict__ idx, uint64_t m, uint32_t* __restrict__ deg)
{
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&deg[idx[e]], 1u);
}

static __global__ void k_hot_hist(uint32_t n, const uint32_t* __restrict__ deg, uint32_t* __restrict__ bins)
{
    __shared__ uint32_t h[kHotBins];
    for (uint32_t i = threadIdx.x; i < kHotBins; i += blockDim.x) h[i] = 0u;
    __syncthreads();
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const uint32_t d = deg[u];
        if (d > 1u) atomicAdd(&h[hot_bin(d)], 1u);  // in-degree 0 or 1: never hot
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kHotBins; i += blockDim.x)
        if (h[i]) atomicAdd(&bins[i], h[i]);
}

// deg[u] -> 1 when u is hot, else 0 (in place)
static __global__ void k_hot_flags(uint32_t n, uint32_t* __restrict__ deg, uint32_t thr)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) deg[u] = deg[u] >= thr ? 1u : 0u;
}

// flag -> code (slot of a hot node, ~0 otherwise; in place), hot_node[slot] = u
static __global__ void k_hot_assign(uint32_t n, uint32_t* __restrict__ code, const uint32_t* __restrict__ slot,
                                    uint32_t* __restrict__ hot_node)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    if (code[u]) {
        const uint32_t s = slot[u];
        hot_node[s] = u;
        code[u] = s;
    } else {
        code[u] = ~0u;
    }
}

static __global__ void k_hot_encode(const uint32_t* __restrict__ idx, uint64_t m, const uint32_t* __restrict__ code,
                                    uint32_t* __restrict__ out)
{
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = idx[e];
        const uint32_t c = code[v];
        out[e] = c != ~0u ? (kHotFlag | c) : v;
    }
}

// hot_rank[s] = rank[hot_node[s]] for the hot slots, 0 up to the padded size
static __global__ void k_hot_ranks(uint32_t hot_n, uint32_t padded, const uint32_t* __restrict__ hot_node,
                                   const uint8_t* __restrict__ rank, uint8_t* __restrict__ hot_rank)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < padded) hot_rank[s] = s < hot_n ? rank[hot_node[s]] : (uint8_t)0;
}

// The first signature pass with hot heads.  hot_bytes: the staged table
// (a multiple of 16, the dynamic shared memory of the launch).
template <bool WEIGHTED>
static __global__ void __launch_bounds__(kHotThreads, 1)
    k_signature_hot(const ActiveSet* __restrict__ as, const RoundState* __restrict__ st, const uint8_t* __restrict__ rank,
                    const uint32_t* __restrict__ hot_idx, const uint8_t* __restrict__ hot_rank, uint32_t hot_bytes,
                    Sig* __restrict__ sig)
{
    extern __shared__ __align__(16) uint8_t s_hot[];
    const uint4* __restrict__ src = reinterpret_cast<const uint4*>(hot_rank);
    uint4* dst = reinterpret_cast<uint4*>(s_hot);
    for (uint32_t i = threadIdx.x; i < hot_bytes / 16u; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    signature_body<WEIGHTED, uint8_t, true, false, true, kHotThreads / 32>(
        as, st, rank, sig, TileRange{0u, 0u, nullptr, nullptr, 0ull}, hot_idx, s_hot);
}

}  // namespace rbsc
