// common.cuh -- shared constants, hash functions and small device helpers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rbsc {

// Colour words: bits 0..30 = label (smallest node id of the block),
// bit 31 = the block is a singleton.  Singleton blocks never split again, so
// their nodes skip the relabel table.
constexpr uint32_t kSingleton = 0x80000000u;
constexpr uint32_t kLabelMask = 0x7fffffffu;
// Relabel-table value word: bits 0..30 = smallest member, bit 31 = the key was
// seen from more than one node (block is not a singleton).
constexpr uint32_t kJoined = 0x80000000u;

// Signature tiles: one warp per tile of 512 arcs, 16 consecutive arcs per lane;
// CTAs of 8 warps.
constexpr int kTileThreads = 256;
constexpr int kEdgesPerThread = 16;
constexpr uint32_t kTileEdges = 32 * kEdgesPerThread;  // 512

constexpr int kNodeThreads = 256;

constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

// MurmurHash3 64-bit finaliser (Austin Appleby, public domain): a bijection
// on uint64 with full avalanche.  Used as the per-arc term of the signature.
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// MurmurHash3 32-bit finaliser (same source): second, independent term.
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// Per-pass salts.  Pass r hashes colour c as fmix64(c ^ salt1(r)) and
// fmix32(c ^ salt2(r)); a fresh salt per pass decorrelates the passes.
__host__ __device__ __forceinline__ uint64_t pass_salt1(uint64_t seed, uint32_t r)
{
    return fmix64(seed + (uint64_t)(r + 1) * kGolden);
}
__host__ __device__ __forceinline__ uint32_t pass_salt2(uint64_t seed, uint32_t r)
{
    return (uint32_t)(fmix64(~seed + (uint64_t)(r + 7) * 0xd1b54a32d192ed03ull) >> 32);
}

template <typename T> __host__ __device__ __forceinline__ T ceil_div(T a, T b) { return (a + b - 1) / b; }

// Block-wide reservation in an output list: every thread with `take` gets a
// distinct position; the block makes one atomicAdd on `counter` (a global
// counter shared by all blocks), instead of one per warp.  Must be called by
// all threads of the block (it synchronises twice).  BLOCK = threads per block.
template <int BLOCK> struct BlockReserveSmem {
    uint32_t warp_pre[BLOCK / 32];
    unsigned long long base;
};

template <int BLOCK>
__device__ __forceinline__ uint32_t block_reserve(bool take, uint32_t* counter, BlockReserveSmem<BLOCK>& sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (lane == 0) sm.warp_pre[warp] = (uint32_t)__popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < BLOCK / 32; ++w) {
            const uint32_t c = sm.warp_pre[w];
            sm.warp_pre[w] = run;
            run += c;
        }
        sm.base = run ? atomicAdd(counter, run) : 0u;
    }
    __syncthreads();
    const uint32_t pos = (uint32_t)sm.base + sm.warp_pre[warp] + (uint32_t)__popc(m & ((1u << lane) - 1u));
    __syncthreads();
    return pos;
}

// Like block_reserve, with `cnt` positions per thread: returns the first of
// the thread's cnt consecutive positions.  Block-collective.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_reserve_n(uint32_t cnt, uint32_t* counter, BlockReserveSmem<BLOCK>& sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) sm.warp_pre[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < BLOCK / 32; ++w) {
            const uint32_t c = sm.warp_pre[w];
            sm.warp_pre[w] = run;
            run += c;
        }
        sm.base = run ? atomicAdd(counter, run) : 0u;
    }
    __syncthreads();
    const uint32_t pos = (uint32_t)sm.base + sm.warp_pre[warp] + incl - cnt;
    __syncthreads();
    return pos;
}

// Sum over the block of a per-thread count, added to `counter` with one
// atomic per block.  Called by all threads of the block.
template <int BLOCK>
__device__ __forceinline__ void block_count(uint32_t v, uint32_t* counter, BlockReserveSmem<BLOCK>& sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = __reduce_add_sync(0xffffffffu, v);
    if (lane == 0) sm.warp_pre[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < BLOCK / 32; ++w) run += sm.warp_pre[w];
        if (run) atomicAdd(counter, run);
    }
    __syncthreads();
}

// Buffered append to a global list: the flagged values of each block
// iteration go to a shared-memory buffer, and the block reserves space in the
// global list (one atomicAdd on the shared counter) only when the buffer is
// full and at the end.  A counter that every block of a large grid hits once
// per iteration serialises in L2 (one atomic after another on one address);
// this makes it one per CAP values.  All calls are block-collective.
template <typename T, int CAP, int BLOCK> struct BlockAppend {
    static_assert(CAP >= BLOCK, "a block iteration must fit in an empty buffer");
    T buf[CAP];
    uint32_t warp_cnt[BLOCK / 32];
    uint32_t count;
    uint32_t base;
};

template <typename T, int CAP, int BLOCK>
__device__ __forceinline__ void block_append_begin(BlockAppend<T, CAP, BLOCK>& s)
{
    if (threadIdx.x == 0) s.count = 0;
    __syncthreads();
}

// Writes the buffered values out (block-collective).
template <typename T, int CAP, int BLOCK>
__device__ __forceinline__ void block_append_flush(BlockAppend<T, CAP, BLOCK>& s, uint32_t* counter, T* out)
{
    __syncthreads();
    const uint32_t cnt = s.count;
    if (cnt == 0) return;
    if (threadIdx.x == 0) s.base = atomicAdd(counter, cnt);
    __syncthreads();
    const uint32_t base = s.base;
    for (uint32_t i = threadIdx.x; i < cnt; i += BLOCK) out[base + i] = s.buf[i];
    __syncthreads();
    if (threadIdx.x == 0) s.count = 0;
    __syncthreads();
}

template <typename T, int CAP, int BLOCK>
__device__ __forceinline__ void block_append(BlockAppend<T, CAP, BLOCK>& s, bool take, const T& v, uint32_t* counter, T* out)
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (lane == 0) s.warp_cnt[warp] = (uint32_t)__popc(m);
    __syncthreads();
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < BLOCK / 32; ++w) {
        const uint32_t c = s.warp_cnt[w];
        before += (w < (int)warp) ? c : 0u;
        total += c;
    }
    uint32_t cnt = s.count;
    if (cnt + total > (uint32_t)CAP) {  // block-uniform
        block_append_flush(s, counter, out);
        cnt = 0;
    }
    if (take) s.buf[cnt + before + (uint32_t)__popc(m & ((1u << lane) - 1u))] = v;
    __syncthreads();
    if (threadIdx.x == 0) s.count = cnt + total;
}

// Warp-private buffered append: a warp gathers its flagged values in a
// shared-memory buffer of kWarpBuf entries and reserves space in the global
// list (one atomicAdd by lane 0) only when the buffer could overflow and at
// the end.  No block barrier: only the warp's own lanes take part, so it
// costs a ballot and a few shuffles per call where BlockAppend costs two
// block-wide barriers.  Calls are warp-collective (all 32 lanes).
constexpr uint32_t kWarpBuf = 256;

template <typename T>
__device__ __forceinline__ void warp_append_flush(T* buf, uint32_t& cnt, uint32_t* counter, T* out)
{
    __syncwarp();
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0 && cnt) base = atomicAdd(counter, cnt);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane; i < cnt; i += 32) out[base + i] = buf[i];
    __syncwarp();
    cnt = 0;
}

template <typename T>
__device__ __forceinline__ void warp_append(bool take, const T& v, T* buf, uint32_t& cnt, uint32_t* counter, T* out)
{
    const uint32_t lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    if (cnt + 32u > kWarpBuf) warp_append_flush(buf, cnt, counter, out);  // warp-uniform
    if (take) buf[cnt + (uint32_t)__popc(m & ((1u << lane) - 1u))] = v;
    cnt += (uint32_t)__popc(m);
}

// Kernels enqueued by the calling host thread (reported in rbsc_stats).
inline uint64_t& launch_counter()
{
    static thread_local uint64_t c = 0;
    return c;
}

}  // namespace rbsc
