// prep_kernels.cuh -- one-time per-graph preparation of the signature tiling.
//
// The reference feeds CUB a COO edge list (edge_start, edge_end, weight; 16 B
// per arc, rbsc.cu:341-344).  Here the resident graph is CSR plus, built once:
//   rows[k]      node id of the k-th non-empty row
//   roff[k]      first arc of that row (uint32 when M < 2^32), roff[K] = M
//   tile_row[t]  the non-empty row holding arc t*2048, tile_row[ntiles] = K
//   split[]      rows whose arcs span more than one tile (their signatures are
//                accumulated atomically and zeroed between passes)
// Rows without arcs never enter the signature pass: their signature is the
// empty sum, 0, for good.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace rbsc {

static __global__ void k_validate(uint32_t n, uint64_t m, const uint64_t* __restrict__ off, const uint32_t* __restrict__ idx,
                           uint32_t* __restrict__ err)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        if (off[i] > off[i + 1]) atomicOr(err, 1u);
    }
    if (i == 0 && (off[0] != 0 || off[n] != m)) atomicOr(err, 2u);
    if (idx)  // null: the heads are checked as they arrive (k_validate_heads)
        for (uint64_t k = i; k < m; k += (uint64_t)gridDim.x * blockDim.x)
            if (idx[k] >= n) atomicOr(err, 4u);
}

template <typename OffIn>
static __global__ void k_widen_offsets(uint64_t count, const OffIn* __restrict__ in, uint64_t* __restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (uint64_t)in[i];
}

static __global__ void k_nonempty_flags(uint32_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ flag)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) flag[u] = off[u + 1] > off[u] ? 1u : 0u;
}

template <typename OffT>
static __global__ void k_prep_rows(uint32_t n, uint64_t m, const uint64_t* __restrict__ off, const uint32_t* __restrict__ pos,
                               uint32_t K, uint32_t* __restrict__ rows, OffT* __restrict__ roff)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n && off[u + 1] > off[u]) {
        const uint32_t k = pos[u];
        rows[k] = u;
        roff[k] = (OffT)off[u];
    }
    if (u == 0) roff[K] = (OffT)m;
}

template <typename OffT>
static __global__ void k_tile_rows(uint32_t ntiles, uint32_t K, const OffT* __restrict__ roff, uint32_t* __restrict__ tile_row)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    if (t == ntiles) {
        tile_row[t] = K;
        return;
    }
    const uint64_t e = (uint64_t)t * kTileEdges;
    // largest k < K with roff[k] <= e
    uint32_t lo = 0, hi = K - 1;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo + 1) >> 1);
        if ((uint64_t)roff[mid] <= e) lo = mid; else hi = mid - 1;
    }
    tile_row[t] = lo;
}

template <typename OffT>
static __global__ void k_split_flags(uint32_t K, const OffT* __restrict__ roff, uint32_t* __restrict__ flag)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) flag[k] = ((uint64_t)roff[k] / kTileEdges) != (((uint64_t)roff[k + 1] - 1) / kTileEdges) ? 1u : 0u;
}

template <typename OffT>
static __global__ void k_split_compact(uint32_t K, const OffT* __restrict__ roff, const uint32_t* __restrict__ rows,
                                const uint32_t* __restrict__ pos, uint32_t* __restrict__ split)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K && ((uint64_t)roff[k] / kTileEdges) != (((uint64_t)roff[k + 1] - 1) / kTileEdges)) split[pos[k]] = rows[k];
}

}  // namespace rbsc
