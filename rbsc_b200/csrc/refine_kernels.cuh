// refine_kernels.cuh -- the per-round kernels of the colour-refinement loop.
//
// One pass (reference: the body of the round loop, src/rbsc/rbsc.cu:354-425):
//   k_signature  sig(u) = sum over u's arcs of wt * H(colour(v))      (rbsc.cu:80-87 + ReduceByKey 366-382)
//   k_insert     (colour(u), sig(u)) -> relabel-table slot             (replaces the sorts + scan of 384-396)
//   k_relabel    new colour = smallest member of the slot's class      (replaces reorder 396)
//   k_fixpoint   block count unchanged -> done                          (replaces the D2H + host test of 398-402, 425)
// The reference's injectivity loop (rbsc.cu:404-419) has no counterpart: the
// per-arc hash here is a bijection of the colour by construction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace rbsc {

constexpr int kRoundLog = 64;

// Device-resident loop state; every kernel of a pass reads it, only
// k_fixpoint (one thread) advances it.
struct RoundState {
    uint32_t round;          // completed signature passes
    uint32_t parity;         // colour buffer holding the current colouring
    uint32_t count;          // blocks counted by the running pass
    uint32_t prev;           // blocks after the last completed pass
    uint32_t done;           // fixpoint reached
    uint32_t error;          // device error bits (kErr*)
    uint32_t max_rounds;
    uint32_t stamp;          // relabel-table stamp of the running pass, 1..255
    uint32_t clear_pending;  // table must be cleared before the running pass
    uint32_t hash_bits;      // test hook: signatures truncated to this many bits (0 = off)
    uint64_t seed;
    uint32_t round_blocks[kRoundLog];
};

constexpr uint32_t kErrProbe = 1u;   // relabel table full (cannot happen at load <= 1/2)
constexpr uint32_t kErrRounds = 2u;  // max_rounds reached

// Pass modes of k_insert / k_fixpoint.
constexpr int kModeHash = 0;    // key = (label, signature)
constexpr int kModeInit = 1;    // key = initial colour (exact)
constexpr int kModeRepair = 2;  // key = (label, failed-exact-check flag) (exact)

// ---------------------------------------------------------------------------
// relabel table: 16-byte entries {k1 (64), k2 (32: 24 hash bits | 8-bit stamp),
// val (32: smallest member | kJoined)}.  An entry whose stamp differs from the
// running pass is empty for that pass, so the table is cleared only when the
// 8-bit stamp wraps (every 255 passes).
// ---------------------------------------------------------------------------
struct __align__(16) Entry {
    unsigned long long k1;
    unsigned long long hi;  // (val << 32) | k2
};

__device__ __forceinline__ void ld_entry(const Entry* p, uint64_t& lo, uint64_t& hi)
{
    asm volatile("{\n\t.reg .b128 t;\n\tld.relaxed.gpu.global.b128 t, [%2];\n\tmov.b128 {%0, %1}, t;\n\t}"
                 : "=l"(lo), "=l"(hi)
                 : "l"(p)
                 : "memory");
}

__device__ __forceinline__ void cas_entry(Entry* p, uint64_t clo, uint64_t chi, uint64_t nlo, uint64_t nhi, uint64_t& olo,
                                          uint64_t& ohi)
{
    asm volatile(
        "{\n\t.reg .b128 c, n, d;\n\tmov.b128 c, {%2, %3};\n\tmov.b128 n, {%4, %5};\n\t"
        "atom.relaxed.gpu.global.cas.b128 d, [%6], c, n;\n\tmov.b128 {%0, %1}, d;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(nlo), "l"(nhi), "l"(p)
        : "memory");
}

// Finds or claims the slot of key (k1, k2) for node u.  `multi`: u stands for
// several nodes with this key (warp-aggregated), so the class is not a
// singleton.  Returns the slot; *claimed = this call created the class.
__device__ __forceinline__ uint32_t table_insert(Entry* tab, uint32_t log2size, uint64_t k1, uint32_t k2, uint32_t stamp,
                                                 uint32_t u, bool multi, bool* claimed, uint32_t* err)
{
    const uint32_t mask = (1u << log2size) - 1u;
    uint32_t s = (uint32_t)((k1 * kGolden + k2) >> (64 - log2size)) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        uint64_t lo, hi;
        ld_entry(tab + s, lo, hi);
        if (((uint32_t)hi & 0xffu) != stamp) {
            const uint64_t nhi = ((uint64_t)(u | (multi ? kJoined : 0u)) << 32) | k2;
            uint64_t olo, ohi;
            cas_entry(tab + s, lo, hi, k1, nhi, olo, ohi);
            if (olo == lo && ohi == hi) {
                *claimed = true;
                return s;
            }
            lo = olo;  // claimed by another node during this pass
            hi = ohi;
        }
        if (lo == k1 && (uint32_t)hi == k2) {
            const uint32_t v = (uint32_t)(hi >> 32);
            if (!(v & kJoined) || (v & kLabelMask) > u) {
                uint32_t* vp = reinterpret_cast<uint32_t*>(tab + s) + 3;
                atomicOr(vp, kJoined);
                atomicMin(vp, u | kJoined);
            }
            *claimed = false;
            return s;
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, kErrProbe);
    *claimed = false;
    return 0;
}

// ---------------------------------------------------------------------------
// Per-arc term of the signature: an injective function of the head colour c
// (the multiply by an odd constant, the xor-shift and the second multiply are
// all bijections of uint64), salted per pass.  t1 feeds the 64-bit sum, t2 a
// second, independent-looking 32-bit sum.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void arc_terms(uint32_t c, uint64_t salt, uint64_t& t1, uint32_t& t2)
{
    uint64_t y = (uint64_t)(c ^ (uint32_t)salt) * 0x9e3779b97f4a7c15ull;
    y ^= y >> 32;
    y *= 0xd6e8feb86659fd93ull;
    y ^= y >> 32;
    t1 = y + (salt >> 32);
    t2 = (uint32_t)(y >> 32) * 0x2545f491u + (uint32_t)y * ((uint32_t)y | 1u);
}

// Block-wide scans over the 256 threads of a tile CTA.
struct TileScanSmem {
    uint32_t heads[kTileThreads / 32];
    uint32_t flag[kTileThreads / 32];
    unsigned long long v1[kTileThreads / 32];
    uint32_t v2[kTileThreads / 32];
    unsigned long long c1[kTileThreads];
    uint32_t c2[kTileThreads];
};

// exclusive prefix over the block of n (per thread)
__device__ __forceinline__ uint32_t tile_excl_scan(TileScanSmem& sm, uint32_t n)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t h = n;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, h, d);
        if (lane >= d) h += o;
    }
    if (lane == 31) sm.heads[warp] = h;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < warp; ++w) base += sm.heads[w];
    return base + h - n;
}

// inclusive segmented prefix of (v1, v2) over the block, a segment starting at
// every thread whose flag is set; also returns the previous thread's result
// (cin), i.e. what arrives at this thread's first arc
__device__ __forceinline__ void tile_seg_scan(TileScanSmem& sm, bool flag, uint64_t v1, uint32_t v2, uint64_t& c1,
                                              uint32_t& c2, uint64_t& cin1, uint32_t& cin2)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t f = flag ? 1u : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t fo = __shfl_up_sync(0xffffffffu, f, d);
        const uint64_t vo1 = __shfl_up_sync(0xffffffffu, v1, d);
        const uint32_t vo2 = __shfl_up_sync(0xffffffffu, v2, d);
        if (lane >= d) {
            if (!f) {
                v1 += vo1;
                v2 += vo2;
            }
            f |= fo;
        }
    }
    if (lane == 31) {
        sm.flag[warp] = f;
        sm.v1[warp] = v1;
        sm.v2[warp] = v2;
    }
    __syncthreads();
    if (!f) {
        uint64_t cc1 = 0;
        uint32_t cc2 = 0;
        for (int w = 0; w < warp; ++w) {
            if (sm.flag[w]) {
                cc1 = sm.v1[w];
                cc2 = sm.v2[w];
            } else {
                cc1 += sm.v1[w];
                cc2 += sm.v2[w];
            }
        }
        v1 += cc1;
        v2 += cc2;
    }
    c1 = v1;
    c2 = v2;
    sm.c1[threadIdx.x] = c1;
    sm.c2[threadIdx.x] = c2;
    __syncthreads();
    cin1 = threadIdx.x ? sm.c1[threadIdx.x - 1] : 0ull;
    cin2 = threadIdx.x ? sm.c2[threadIdx.x - 1] : 0u;
}

// ---------------------------------------------------------------------------
// k_signature: edge-balanced tiles.  Tile t holds arcs [t*2048, (t+1)*2048);
// thread i of the tile CTA owns the 8 consecutive arcs [8i, 8i+8): two 16-byte
// loads of heads, one byte of the row-head bitmap (bit j set = arc 8i+j starts
// a row), 8 gathered head colours.  An exclusive scan of the head counts gives
// every thread the index of its first row.  Each thread then folds its arcs:
//   - rows that start and end inside its 8 arcs are written directly,
//   - the part before its first head belongs to the row continuing from the
//     previous thread, the part after its last head to the row continuing into
//     the next thread;
// a block-wide segmented scan joins the parts of rows that span threads, and
// the thread in which such a row ends writes it.  A row that crosses a tile
// edge is added to global memory atomically (its signature was zeroed by the
// previous pass).  Sums are modulo 2^64 / 2^32, so the split into partial sums
// does not change the result.  No shared-memory atomics.
// ---------------------------------------------------------------------------
template <bool WEIGHTED>
static __global__ void __launch_bounds__(kTileThreads) k_signature(const uint32_t* __restrict__ rows,
                                                                   const uint32_t* __restrict__ tile_row,
                                                                   const uint8_t* __restrict__ head8,
                                                                   const uint32_t* __restrict__ idx,
                                                                   const uint64_t* __restrict__ wt, uint64_t m,
                                                                   const RoundState* __restrict__ st,
                                                                   const uint32_t* __restrict__ col0,
                                                                   const uint32_t* __restrict__ col1,
                                                                   unsigned long long* __restrict__ sig1,
                                                                   uint32_t* __restrict__ sig2)
{
    __shared__ TileScanSmem sm;
    const uint32_t* __restrict__ col = st->parity ? col1 : col0;
    const uint64_t salt = pass_salt1(st->seed, st->round);

    const uint64_t tbeg = (uint64_t)blockIdx.x * kTileEdges;
    const uint32_t tlen = (uint32_t)min((uint64_t)kTileEdges, m - tbeg);
    const uint64_t tend = tbeg + tlen;
    const uint32_t k0 = tile_row[blockIdx.x];
    const uint32_t h0 = head8[tbeg >> 3] & 1u;  // the tile's first arc starts a row
    const uint32_t a = threadIdx.x * kEdgesPerThread;
    const uint32_t cnt = a < tlen ? min((uint32_t)kEdgesPerThread, tlen - a) : 0u;

    uint32_t hb = 0;
    uint32_t v[kEdgesPerThread];
    if (cnt == kEdgesPerThread) {
        hb = head8[(tbeg + a) >> 3];
        const uint4* p = reinterpret_cast<const uint4*>(idx + tbeg + a);
        const uint4 q0 = __ldcs(p), q1 = __ldcs(p + 1);
        v[0] = q0.x; v[1] = q0.y; v[2] = q0.z; v[3] = q0.w;
        v[4] = q1.x; v[5] = q1.y; v[6] = q1.z; v[7] = q1.w;
    } else {
        if (cnt) hb = head8[(tbeg + a) >> 3] & ((1u << cnt) - 1u);
#pragma unroll
        for (int i = 0; i < kEdgesPerThread; ++i) v[i] = (uint32_t)i < cnt ? __ldcs(idx + tbeg + a + i) : 0u;
    }
    uint32_t c[kEdgesPerThread];
#pragma unroll
    for (int i = 0; i < kEdgesPerThread; ++i) c[i] = (uint32_t)i < cnt ? __ldg(col + v[i]) : 0u;
    uint64_t w[kEdgesPerThread];
    if (WEIGHTED) {
#pragma unroll
        for (int i = 0; i < kEdgesPerThread; ++i) w[i] = (uint32_t)i < cnt ? __ldcs(wt + tbeg + a + i) : 0ull;
    }

    // row of arc a-1 (or of arc a when arc a does not start a row):
    // k0 + (heads in tile arcs [0, a)) - h0
    const uint32_t kbase = k0 + tile_excl_scan(sm, (uint32_t)__popc(hb)) - h0;

    // fold: `pre` = arcs before this thread's first head, `cur` = the row
    // opened by the latest head; a row closed inside the thread is written
    uint64_t pre1 = 0, cur1 = 0;
    uint32_t pre2 = 0, cur2 = 0;
    uint32_t nh = 0;
#pragma unroll
    for (int i = 0; i < kEdgesPerThread; ++i) {
        if ((uint32_t)i < cnt) {
            if ((hb >> i) & 1u) {
                if (nh > 0) {
                    const uint32_t node = rows[kbase + nh];
                    sig1[node] = cur1;
                    sig2[node] = cur2;
                }
                ++nh;
                cur1 = 0;
                cur2 = 0;
            }
            uint64_t t1;
            uint32_t t2;
            arc_terms(c[i], salt, t1, t2);
            if (WEIGHTED) {
                t1 *= w[i];
                t2 *= (uint32_t)w[i];
            }
            if (nh == 0) {
                pre1 += t1;
                pre2 += t2;
            } else {
                cur1 += t1;
                cur2 += t2;
            }
        }
    }

    uint64_t c1, cin1;
    uint32_t c2, cin2;
    const bool flag = nh > 0;
    tile_seg_scan(sm, flag, flag ? cur1 : pre1, flag ? cur2 : pre2, c1, c2, cin1, cin2);
    if (cnt == 0) return;

    // the row continuing into this thread ends here when this thread has a head
    if (nh > 0 && (a > 0 || !(hb & 1u))) {
        const uint32_t node = rows[kbase];
        const uint64_t tot1 = cin1 + pre1;
        const uint32_t tot2 = cin2 + pre2;
        if (kbase == k0 && !h0) {  // began in an earlier tile
            atomicAdd(&sig1[node], (unsigned long long)tot1);
            atomicAdd(&sig2[node], tot2);
        } else {
            sig1[node] = tot1;
            sig2[node] = tot2;
        }
    }
    // the last thread of the tile closes the tile's last row
    if (a + cnt == tlen) {
        const uint32_t klast = kbase + nh;
        const bool ends = (tend == m) || (head8[tend >> 3] & 1u);
        const bool began_before = (klast == k0 && !h0);
        const uint32_t node = rows[klast];
        if (ends && !began_before) {
            sig1[node] = c1;
            sig2[node] = c2;
        } else {
            atomicAdd(&sig1[node], (unsigned long long)c1);
            atomicAdd(&sig2[node], c2);
        }
    }
}

// Row-head bitmap: bit (e % 8) of byte e / 8 is set iff arc e is the first
// arc of its row.
template <typename OffT>
static __global__ void k_head_bits(uint32_t K, const OffT* __restrict__ roff, uint32_t* __restrict__ head32)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) {
        const uint64_t e = (uint64_t)roff[k];
        atomicOr(&head32[e >> 5], 1u << (e & 31));
    }
}

// ---------------------------------------------------------------------------
// k_insert: one thread per node.  Singleton nodes keep their colour.  The
// others build their key, group with equal keys of their warp
// (__match_any_sync), and the group's smallest node probes the table once for
// the group.  Counts the blocks of the new partition.
// ---------------------------------------------------------------------------
template <int MODE>
static __global__ void __launch_bounds__(kNodeThreads) k_insert(uint32_t n, RoundState* __restrict__ st,
                                                         const uint32_t* __restrict__ col0, const uint32_t* __restrict__ col1,
                                                         const unsigned long long* __restrict__ sig1,
                                                         const uint32_t* __restrict__ sig2,
                                                         const uint32_t* __restrict__ aux, Entry* __restrict__ tab,
                                                         uint32_t log2size, uint32_t* __restrict__ slot)
{
    const uint32_t u = blockIdx.x * kNodeThreads + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool active = u < n;
    const uint32_t* __restrict__ col = st->parity ? col1 : col0;
    const uint32_t stamp = st->stamp;
    const uint32_t c = active ? col[u] : kSingleton;
    const bool need = active && (MODE == kModeInit || !(c & kSingleton));

    uint64_t k1 = 0;
    uint32_t k2 = stamp;
    if (need) {
        const uint32_t lab = c & kLabelMask;
        if (MODE == kModeHash) {
            uint64_t s1 = sig1[u];
            uint32_t s2 = sig2[u];
            const uint32_t hb = st->hash_bits;
            if (hb) {
                s1 &= (hb >= 64) ? ~0ull : ((1ull << hb) - 1ull);
                s2 = 0;
            }
            const uint64_t seed = st->seed;
            k1 = s1 ^ fmix64(((uint64_t)lab << 1 | 1ull) * kGolden ^ seed);
            k2 = ((s2 ^ fmix32(lab * 0x9e3779b1u + (uint32_t)seed)) & 0xffffff00u) | stamp;
        } else if (MODE == kModeInit) {
            k1 = aux[u];
        } else {
            k1 = (uint64_t)lab | ((uint64_t)(aux[u] != 0u) << 32);
        }
    }
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    bool new_block = active && !need;
    if (need) {
        const unsigned peers = __match_any_sync(need_mask, k1) & __match_any_sync(need_mask, k2);
        const int leader = __ffs(peers) - 1;
        uint32_t s = 0;
        bool claimed = false;
        if (lane == leader) s = table_insert(tab, log2size, k1, k2, stamp, u, __popc(peers) > 1, &claimed, &st->error);
        s = __shfl_sync(peers, s, leader);
        slot[u] = s;
        new_block = (lane == leader) && claimed;
    }
    const unsigned nb = __ballot_sync(0xffffffffu, new_block);
    if (lane == 0 && nb) atomicAdd(&st->count, (uint32_t)__popc(nb));
}

// k_relabel: new colour of every node; also zeroes the signatures of the rows
// that cross a tile edge (the next pass adds into them atomically).
static __global__ void __launch_bounds__(kNodeThreads) k_relabel(uint32_t n, const RoundState* __restrict__ st, uint32_t* __restrict__ col0,
                                                          uint32_t* __restrict__ col1, const Entry* __restrict__ tab,
                                                          const uint32_t* __restrict__ slot,
                                                          const uint32_t* __restrict__ split_rows, uint32_t nsplit,
                                                          unsigned long long* __restrict__ sig1, uint32_t* __restrict__ sig2)
{
    const uint32_t u = blockIdx.x * kNodeThreads + threadIdx.x;
    const uint32_t* __restrict__ cur = st->parity ? col1 : col0;
    uint32_t* __restrict__ nxt = st->parity ? col0 : col1;
    if (u < n) {
        const uint32_t c = cur[u];
        uint32_t out = c;
        if (!(c & kSingleton)) {
            const uint32_t v = __ldcg(reinterpret_cast<const uint32_t*>(tab + slot[u]) + 3);
            out = (v & kLabelMask) | ((v & kJoined) ? 0u : kSingleton);
        }
        nxt[u] = out;
    }
    for (uint32_t i = u; i < nsplit; i += gridDim.x * kNodeThreads) {
        const uint32_t node = split_rows[i];
        sig1[node] = 0ull;
        sig2[node] = 0u;
    }
}

// k_fixpoint: one thread.  Closes the running pass and decides whether the
// device-side while loop runs another one.
template <int MODE>
static __global__ void k_fixpoint(RoundState* st, cudaGraphConditionalHandle handle, int use_handle)
{
    const uint32_t cnt = st->count;
    st->count = 0;
    if (MODE == kModeHash) {
        const uint32_t r = st->round + 1u;
        st->round = r;
        if (r < kRoundLog) st->round_blocks[r] = cnt;
        if (cnt == st->prev) st->done = 1u;
    } else if (MODE == kModeInit) {
        st->round_blocks[0] = cnt;
        st->done = 0u;
    } else {
        st->done = 0u;
    }
    st->prev = cnt;
    st->parity ^= 1u;
    const uint32_t stamp = st->stamp % 255u + 1u;
    st->stamp = stamp;
    st->clear_pending = stamp == 1u;
    if (!st->done && st->round >= st->max_rounds) st->error |= kErrRounds;
    const bool more = !st->done && !st->error;
    if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// k_clear_table: clears the table when the stamp wrapped.
static __global__ void k_clear_table(const RoundState* __restrict__ st, Entry* __restrict__ tab, uint64_t entries)
{
    if (!st->clear_pending) return;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += (uint64_t)gridDim.x * blockDim.x) {
        tab[i].k1 = 0ull;
        tab[i].hi = 0ull;
    }
}

// One initial block for every node: colour 0, singleton iff n == 1.
static __global__ void k_fill_uniform(uint32_t n, uint32_t* __restrict__ col)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) col[u] = (n == 1u) ? kSingleton : 0u;
}

// floor(log2(deg + 1)) from per-node offsets.
static __global__ void k_degree_colors(uint32_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ out)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) {
        const uint64_t d = off[u + 1] - off[u] + 1ull;
        out[u] = 63u - (uint32_t)__clzll((long long)d);
    }
}

// Canonical labels out of colour words.
static __global__ void k_strip_labels(uint32_t n, const uint32_t* __restrict__ col, uint32_t* __restrict__ out)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) out[u] = col[u] & kLabelMask;
}

}  // namespace rbsc
