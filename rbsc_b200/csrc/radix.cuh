// radix.cuh -- hand-written stable LSD radix sort of uint64 keys with an
// optional value array (8-bit digits, one histogram + one scatter kernel per
// digit).  Replaces the cub::DeviceRadixSort calls of src/rbsc/rbsc.cu:386-390
// and 409 where this implementation still sorts: the exact collision check,
// the sort-based relabel mode and the R-MAT generator's duplicate removal.
//
// Per pass: k_rs_hist counts the digits of a tile of 4096 keys per CTA into
// hist[digit][tile]; an exclusive scan over that digit-major array gives every
// (digit, tile) its output base; k_rs_scatter re-reads the tile and writes each
// key to base + its stable rank.  Stability inside a tile: warp w owns keys
// [w*512, (w+1)*512) of the tile, walks them 32 at a time in memory order, and
// ranks equal digits with __match_any_sync.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "scan.cuh"

namespace rbsc {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsIters = 16;                                  // keys per lane
constexpr uint64_t kRsTile = (uint64_t)kRsThreads * kRsIters;  // 4096
constexpr int kRsBins = 256;

static __global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned long long* __restrict__ keys, uint64_t n, int shift,
                                                        uint32_t* __restrict__ hist, uint32_t ntiles)
{
    __shared__ uint32_t s_hist[kRsBins];
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
#pragma unroll 4
    for (int it = 0; it < kRsIters; ++it) {
        const uint64_t i = base + (uint64_t)it * kRsThreads + threadIdx.x;
        const bool valid = i < n;
        const uint32_t d = valid ? (uint32_t)(keys[i] >> shift) & 0xffu : 0u;
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned peers = __match_any_sync(act, d);
            if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&s_hist[d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = s_hist[threadIdx.x];
}

template <typename V, bool HAS_V>
static __global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned long long* __restrict__ keys_in, const V* __restrict__ vals_in,
                                                           unsigned long long* __restrict__ keys_out, V* __restrict__ vals_out, uint64_t n,
                                                           int shift, const uint32_t* __restrict__ hist_scan, uint32_t ntiles)
{
    __shared__ uint32_t s_cnt[kRsWarps][kRsBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRsWarps * kRsBins; i += kRsThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();

    const uint64_t wbase = (uint64_t)blockIdx.x * kRsTile + (uint64_t)warp * (kRsIters * 32);
    unsigned long long k[kRsIters];
    V v[kRsIters];
    uint32_t rank[kRsIters];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kRsIters; ++it) {
        const uint64_t i = wbase + (uint64_t)it * 32 + lane;
        const bool valid = i < n;
        k[it] = valid ? keys_in[i] : ~0ull;
        if (HAS_V) v[it] = valid ? vals_in[i] : V(0);
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        rank[it] = 0;
        if (valid) {
            const uint32_t d = (uint32_t)(k[it] >> shift) & 0xffu;
            const unsigned peers = __match_any_sync(act, d);
            // rank among equal digits of this warp so far; leader bumps the count
            const uint32_t before = s_cnt[warp][d];
            rank[it] = before + __popc(peers & lt);
            __syncwarp(act);
            if (lane == __ffs(peers) - 1) s_cnt[warp][d] = before + __popc(peers);
            __syncwarp(act);
        }
    }
    __syncthreads();
    // per digit: prefix over warps + this tile's global base
    {
        const int d = threadIdx.x;  // kRsThreads == kRsBins
        uint32_t run = hist_scan[(uint64_t)d * ntiles + blockIdx.x];
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) {
            const uint32_t c = s_cnt[w][d];
            s_cnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kRsIters; ++it) {
        const uint64_t i = wbase + (uint64_t)it * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)(k[it] >> shift) & 0xffu;
            const uint32_t pos = s_cnt[warp][d] + rank[it];
            keys_out[pos] = k[it];
            if (HAS_V) vals_out[pos] = v[it];
        }
    }
}

inline size_t radix_temp_bytes(uint64_t n)
{
    const uint64_t tiles = ceil_div<uint64_t>(n ? n : 1, kRsTile);
    const uint64_t h = tiles * kRsBins;
    return ((h * 4 + 255) / 256) * 256 + scan_temp_bytes<uint32_t>(h);
}

// Sorts keys[0..n) on bits [begin_bit, end_bit) (stable), carrying vals when
// non-null.  Ping-pongs between (keys, vals) and (keys_alt, vals_alt); returns
// true when the sorted result ended in the *_alt buffers.  n < 2^32.
template <typename V>
inline cudaError_t radix_sort(unsigned long long* keys, unsigned long long* keys_alt, V* vals, V* vals_alt, uint64_t n, int begin_bit, int end_bit,
                              void* temp, cudaStream_t s, bool* in_alt)
{
    *in_alt = false;
    if (n <= 1 || end_bit <= begin_bit) return cudaSuccess;
    const uint32_t tiles = (uint32_t)ceil_div<uint64_t>(n, kRsTile);
    uint32_t* hist = (uint32_t*)temp;
    void* scan_tmp = (char*)temp + (((uint64_t)tiles * kRsBins * 4 + 255) / 256) * 256;
    unsigned long long *ki = keys, *ko = keys_alt;
    V *vi = vals, *vo = vals_alt;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        ++rbsc::launch_counter();
        k_rs_hist<<<tiles, kRsThreads, 0, s>>>(ki, n, shift, hist, tiles);
        cudaError_t e = exclusive_scan<uint32_t, uint32_t>(hist, hist, (uint64_t)tiles * kRsBins, (uint32_t*)nullptr, scan_tmp, s);
        if (e != cudaSuccess) return e;
        if (vals) {
            ++rbsc::launch_counter();
            k_rs_scatter<V, true><<<tiles, kRsThreads, 0, s>>>(ki, vi, ko, vo, n, shift, hist, tiles);
        }
        else {
            ++rbsc::launch_counter();
            k_rs_scatter<V, false><<<tiles, kRsThreads, 0, s>>>(ki, vi, ko, vo, n, shift, hist, tiles);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        unsigned long long* tk = ki; ki = ko; ko = tk;
        V* tv = vi; vi = vo; vo = tv;
        *in_alt = !*in_alt;
    }
    return cudaSuccess;
}

}  // namespace rbsc
