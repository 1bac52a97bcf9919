// scan.cuh -- device-wide exclusive prefix sum (reduce-then-scan), used for
// compactions, CSR offsets and the radix-sort digit offsets.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace rbsc {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint64_t kScanTile = kScanThreads * kScanItems;  // 2048

template <typename T> __device__ __forceinline__ T warp_incl_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Exclusive scan of one value per thread across the block; returns the
// exclusive prefix and writes the block total to *total.
template <typename T> __device__ __forceinline__ T block_excl_scan(T v, T* total)
{
    __shared__ T s_warp[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanThreads / 32 ? s_warp[lane] : T(0);
        T wi = warp_incl_scan(w);
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) *total = wi;
    }
    __syncthreads();
    T r = s_warp[warp] + inc - v;
    __syncthreads();
    return r;
}

// in -> per-tile sums
template <typename TI, typename TO>
static __global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const TI* __restrict__ in, uint64_t n, TO* __restrict__ part)
{
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    TO s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) s += (TO)in[base + i];
    __shared__ TO total;
    block_excl_scan<TO>(s, &total);
    if (threadIdx.x == 0) part[blockIdx.x] = total;
}

// exclusive scan of each tile, offset by the scanned tile sums (part may be null)
template <typename TI, typename TO>
static __global__ void __launch_bounds__(kScanThreads) k_scan_apply(const TI* __restrict__ in, uint64_t n, const TO* __restrict__ part,
                                                             TO* __restrict__ out, TO* __restrict__ grand_total)
{
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    TO v[kScanItems];
    TO s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? (TO)in[base + i] : TO(0);
        s += v[i];
    }
    __shared__ TO total;
    TO pre = block_excl_scan<TO>(s, &total);
    if (part) pre += part[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
    // the last tile writes the grand total
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *grand_total = pre;
}

// Temporary bytes needed by exclusive_scan for n elements of TO.
template <typename TO> inline size_t scan_temp_bytes(uint64_t n)
{
    size_t bytes = 0;
    uint64_t len = n;
    while (len > kScanTile) {
        len = ceil_div<uint64_t>(len, kScanTile);
        bytes += ((len * sizeof(TO) + 255) / 256) * 256 * 2;
    }
    return bytes + 256;
}

// out[i] = sum(in[0..i-1]); *grand_total (device pointer, may be null) =
// sum of all.  `in` and `out` may alias.  temp: scan_temp_bytes<TO>(n).
template <typename TI, typename TO>
inline cudaError_t exclusive_scan(const TI* in, TO* out, uint64_t n, TO* grand_total, void* temp, cudaStream_t s)
{
    if (n == 0) {
        if (grand_total) return cudaMemsetAsync(grand_total, 0, sizeof(TO), s);
        return cudaSuccess;
    }
    const uint64_t tiles = ceil_div<uint64_t>(n, kScanTile);
    if (tiles == 1) {
        ++rbsc::launch_counter();
        k_scan_apply<TI, TO><<<1, kScanThreads, 0, s>>>(in, n, (const TO*)nullptr, out, grand_total);
        return cudaGetLastError();
    }
    char* t = (char*)temp;
    TO* part = (TO*)t;
    TO* part_scan = (TO*)(t + ((tiles * sizeof(TO) + 255) / 256) * 256);
    char* rest = t + ((tiles * sizeof(TO) + 255) / 256) * 256 * 2;
    ++rbsc::launch_counter();
    k_scan_reduce<TI, TO><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, part);
    cudaError_t e = exclusive_scan<TO, TO>(part, part_scan, tiles, (TO*)nullptr, rest, s);
    if (e != cudaSuccess) return e;
    ++rbsc::launch_counter();
    k_scan_apply<TI, TO><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, part_scan, out, grand_total);
    return cudaGetLastError();
}

}  // namespace rbsc
