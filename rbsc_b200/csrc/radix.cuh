// radix.cuh -- hand-written stable LSD radix sort of uint64 keys with an
// optional value array (8-bit digits, one histogram + one scatter kernel per
// digit).  Replaces the cub::DeviceRadixSort calls of src/rbsc/rbsc.cu:386-390
// and 409 where this implementation still sorts: the exact collision check,
// the sort-based relabel mode and the R-MAT generator's duplicate removal.
//
// Per pass: k_rs_hist counts the digits of a tile of 4096 keys per CTA into
// hist[digit][tile]; an exclusive scan over that digit-major array gives every
// (digit, tile) its output base; k_rs_scatter re-reads the tile, stages it in
// shared memory in digit order and writes each digit's run to its base
// (coalesced stores).  Stability inside a tile: warp w owns keys
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

// The tile's keys are first ranked (stable: the rank of a key among the equal
// digits of its warp, warps in order), then staged in shared memory in digit
// order, then written out from there: consecutive threads write consecutive
// positions of a digit's run, so the stores coalesce (a warp's 32 keys span a
// few runs instead of 32 buckets).  The values follow through the same
// staging buffer.  Keys and values are read from global memory twice (ranking,
// staging); the second read of a 4096-key tile hits L2.  Registers hold only
// the ranks and destinations, so more CTAs fit per SM.
template <typename V, bool HAS_V>
static __global__ void __launch_bounds__(kRsThreads, 4) k_rs_scatter(const unsigned long long* __restrict__ keys_in, const V* __restrict__ vals_in,
                                                           unsigned long long* __restrict__ keys_out, V* __restrict__ vals_out, uint64_t n,
                                                           int shift, const uint32_t* __restrict__ hist_scan, uint32_t ntiles)
{
    __shared__ uint32_t s_cnt[kRsWarps][kRsBins];
    __shared__ uint32_t s_start[kRsBins];  // tile-local start of each digit's run
    __shared__ uint32_t s_base[kRsBins];   // global position of that run
    __shared__ unsigned long long s_stage[kRsTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRsWarps * kRsBins; i += kRsThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();

    const uint64_t tbase = (uint64_t)blockIdx.x * kRsTile;
    const uint32_t cnt = (uint32_t)(n - tbase < kRsTile ? n - tbase : kRsTile);
    const uint64_t wbase = tbase + (uint64_t)warp * (kRsIters * 32);
    uint32_t pos[kRsIters];  // rank among the warp's equal digits, then tile-local position
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kRsIters; ++it) {
        const uint64_t i = wbase + (uint64_t)it * 32 + lane;
        const bool valid = i < n;
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        pos[it] = 0;
        if (valid) {
            const uint32_t d = (uint32_t)(keys_in[i] >> shift) & 0xffu;
            const unsigned peers = __match_any_sync(act, d);
            // rank among equal digits of this warp so far; leader bumps the count
            const uint32_t before = s_cnt[warp][d];
            pos[it] = before + __popc(peers & lt);
            __syncwarp(act);
            if (lane == __ffs(peers) - 1) s_cnt[warp][d] = before + __popc(peers);
            __syncwarp(act);
        }
    }
    __syncthreads();
    // per digit: prefix over warps, the digit's tile-local start and global base
    {
        const int d = threadIdx.x;  // kRsThreads == kRsBins
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) {
            const uint32_t c = s_cnt[w][d];
            s_cnt[w][d] = run;
            run += c;
        }
        uint32_t total;
        s_start[d] = block_excl_scan<uint32_t>(run, &total);
        s_base[d] = hist_scan[(uint64_t)d * ntiles + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kRsIters; ++it) {
        const uint64_t i = wbase + (uint64_t)it * 32 + lane;
        if (i < n) {
            const unsigned long long k = keys_in[i];
            const uint32_t d = (uint32_t)(k >> shift) & 0xffu;
            pos[it] += s_start[d] + s_cnt[warp][d];
            s_stage[pos[it]] = k;
        }
    }
    __syncthreads();
    uint32_t dst[kRsIters];
#pragma unroll
    for (int q = 0; q < kRsIters; ++q) {
        const uint32_t j = (uint32_t)q * kRsThreads + threadIdx.x;
        if (j < cnt) {
            const unsigned long long k = s_stage[j];
            const uint32_t d = (uint32_t)(k >> shift) & 0xffu;
            dst[q] = s_base[d] + (j - s_start[d]);
            keys_out[dst[q]] = k;
        }
    }
    if (HAS_V) {
        V* s_val = reinterpret_cast<V*>(s_stage);
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kRsIters; ++it) {
            const uint64_t i = wbase + (uint64_t)it * 32 + lane;
            if (i < n) s_val[pos[it]] = vals_in[i];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kRsIters; ++q) {
            const uint32_t j = (uint32_t)q * kRsThreads + threadIdx.x;
            if (j < cnt) vals_out[dst[q]] = s_val[j];
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
