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
#include <cuda.h>
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

// ---------------------------------------------------------------------------
// k_signature_hot_tma: the hot first pass with each warp's tile of heads
// brought into shared memory by the tensor memory accelerator instead of
// 16-byte global loads.  The hot-head copy is viewed as a 2-D tensor of
// 128-byte rows (32 heads); one tile (512 arcs) is a 16-row box, loaded with
// the 128-byte swizzle: lane l reads its 16 heads (logical bytes 64l .. 64l+63)
// as four 16-byte words whose physical offsets are the logical ones with bits
// 4-6 XORed by bits 7-9, so the 32 lanes of each read spread over all banks
// (4 wavefronts for 512 bytes).  The loads themselves take no L1 wavefronts.
// One buffer per warp: a lane copies its heads into registers, the warp
// synchronises, and lane 0 asks for the warp's next tile into the same
// buffer, which then arrives while this tile's ranks are gathered and folded.
// Waits are bounded (kErrStage).  Heads beyond the last arc of the last tile
// are loaded from the padded copy and never used.
// ---------------------------------------------------------------------------
constexpr uint32_t kTmaTileBytes = kTileEdges * 4u;  // 2 KB of heads: 16 rows of 128 B

// The heads are read once per pass: the copies carry an evict-first L2
// policy (as the 16-byte loads' .cs), so the stream of heads does not push
// the class ranks and the signatures out of L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap* map, uint32_t row, uint32_t bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(bar), "l"(policy)
        : "memory");
}

template <bool WEIGHTED>
static __global__ void __launch_bounds__(kHotThreads, 1)
    k_signature_hot_tma(const __grid_constant__ CUtensorMap heads, const ActiveSet* __restrict__ as,
                        RoundState* __restrict__ st, const uint8_t* __restrict__ rank,
                        const uint8_t* __restrict__ hot_rank, uint32_t hot_bytes, Sig* __restrict__ sig)
{
    constexpr uint32_t W = kHotThreads / 32;
    extern __shared__ __align__(16) uint8_t s_dyn[];
    __shared__ __align__(8) uint64_t s_bar[W];
    // the staged table, then one 1024-byte aligned 2 KB buffer per warp (the
    // 128-byte swizzle repeats every 1024 bytes of shared memory)
    uint8_t* s_hot = s_dyn;
    const uint32_t dyn = smem_u32(s_dyn);
    const uint32_t stage0 = (dyn + hot_bytes + 1023u) & ~1023u;
    const uint32_t lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t stage = stage0 + wi * kTmaTileBytes;
    const uint8_t* s_stage = s_dyn + (stage - dyn);
    const uint32_t bar = smem_u32(&s_bar[wi]);
    {
        const uint4* __restrict__ src = reinterpret_cast<const uint4*>(hot_rank);
        uint4* dst = reinterpret_cast<uint4*>(s_hot);
        for (uint32_t i = threadIdx.x; i < hot_bytes / 16u; i += blockDim.x) dst[i] = src[i];
    }
    if (lane == 0) {
        mbar_init(&s_bar[wi], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (*(const volatile uint32_t*)&st->error) return;

    const uint32_t ntiles = as->ntiles;
    const uint64_t m = as->m;
    const uint32_t* __restrict__ rows = as->rows;
    const uint32_t* __restrict__ tile_row = as->tile_row;
    const uint8_t* __restrict__ head8 = as->head8;
    const uint64_t* __restrict__ wt = as->wt;
    const uint64_t salt = pass_salt1(st->seed, st->round);
    const uint32_t warps = gridDim.x * W;
    uint32_t tile = blockIdx.x * W + wi;
    const uint64_t policy = l2_evict_first_policy();
    if (tile < ntiles && lane == 0) {
        mbar_expect_tx(&s_bar[wi], kTmaTileBytes);
        tma_load_tile(stage, &heads, tile * 16u, bar, policy);
    }
    // this lane's four 16-byte words of the tile, at their swizzled offsets
    uint32_t off[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t o = lane * 64u + (uint32_t)j * 16u;
        off[j] = o ^ (((o >> 7) & 7u) << 4);
    }
    uint32_t phase = 0;
    for (; tile < ntiles; tile += warps) {
        const bool ok = mbar_wait_bounded(&s_bar[wi], phase);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicOr(&st->error, kErrStage);
            return;
        }
        phase ^= 1u;
        const uint4 q0 = *reinterpret_cast<const uint4*>(s_stage + off[0]);
        const uint4 q1 = *reinterpret_cast<const uint4*>(s_stage + off[1]);
        const uint4 q2 = *reinterpret_cast<const uint4*>(s_stage + off[2]);
        const uint4 q3 = *reinterpret_cast<const uint4*>(s_stage + off[3]);
        __syncwarp();
        const uint32_t next = tile + warps;
        if (next < ntiles && lane == 0) {
            // the generic-proxy reads of the buffer above come before the
            // asynchronous write of the next tile
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&s_bar[wi], kTmaTileBytes);
            tma_load_tile(stage, &heads, next * 16u, bar, policy);
        }
        const uint64_t tbeg = (uint64_t)tile * kTileEdges;
        const uint32_t tlen = (uint32_t)min((uint64_t)kTileEdges, m - tbeg);
        const uint64_t tend = tbeg + tlen;
        const uint32_t k0 = tile_row[tile];
        const uint32_t h0 = head8[tbeg >> 3] & 1u;
        const uint32_t a = lane * kEdgesPerThread;
        const uint32_t cnt = a < tlen ? min((uint32_t)kEdgesPerThread, tlen - a) : 0u;
        uint32_t hb = cnt ? (uint32_t)*reinterpret_cast<const uint16_t*>(head8 + ((tbeg + a) >> 3)) : 0u;
        if (cnt < (uint32_t)kEdgesPerThread) hb &= (1u << cnt) - 1u;
        const uint32_t h[kEdgesPerThread] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w,
                                             q2.x, q2.y, q2.z, q2.w, q3.x, q3.y, q3.z, q3.w};
        uint32_t c[kEdgesPerThread];
        uint64_t w[kEdgesPerThread];
#pragma unroll
        for (int i = 0; i < kEdgesPerThread; ++i)
            c[i] = (uint32_t)i < cnt ? gather_head<true, uint8_t, true>(rank, s_hot, h[i]) : 0u;
        if (WEIGHTED) {
#pragma unroll
            for (int i = 0; i < kEdgesPerThread; ++i) w[i] = (uint32_t)i < cnt ? __ldcs(wt + tbeg + a + i) : 0ull;
        }
        signature_fold<WEIGHTED>(lane, a, cnt, tlen, tend, m, k0, h0, hb, c, w, salt, rows, head8, sig);
    }
}

}  // namespace rbsc
