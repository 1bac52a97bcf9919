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
// k_signature: edge-balanced tiles.  Tile t holds arcs [t*2048, (t+1)*2048);
// thread i of the tile CTA owns 8 consecutive arcs, loads their heads with two
// 16-byte loads, gathers the 8 head colours, hashes them and folds them into
// per-row partial sums.  A row wholly inside one thread's 8 arcs is written
// directly; a row shared by threads goes through a shared-memory accumulator;
// a row that crosses a tile edge is added to global memory atomically (its
// signature was zeroed by the previous pass).  Sums are modulo 2^64 / 2^32, so
// the split into partial sums does not change the result.
// ---------------------------------------------------------------------------
template <typename OffT, bool WEIGHTED>
static __global__ void __launch_bounds__(kTileThreads) k_signature(const OffT* __restrict__ roff, const uint32_t* __restrict__ rows,
                                                            const uint32_t* __restrict__ tile_row,
                                                            const uint32_t* __restrict__ idx,
                                                            const uint64_t* __restrict__ wt, uint64_t m,
                                                            const RoundState* __restrict__ st,
                                                            const uint32_t* __restrict__ col0, const uint32_t* __restrict__ col1,
                                                            unsigned long long* __restrict__ sig1, uint32_t* __restrict__ sig2)
{
    __shared__ uint32_t s_off[kTileEdges + 1];
    __shared__ unsigned long long s_acc1[kTileEdges];
    __shared__ uint32_t s_acc2[kTileEdges];

    const uint32_t r = st->round;
    const uint32_t* __restrict__ col = st->parity ? col1 : col0;
    const uint64_t salt1 = pass_salt1(st->seed, r);
    const uint32_t salt2 = pass_salt2(st->seed, r);

    const uint64_t tbeg = (uint64_t)blockIdx.x * kTileEdges;
    const uint32_t tlen = (uint32_t)min((uint64_t)kTileEdges, m - tbeg);
    const uint64_t tend = tbeg + tlen;
    const uint32_t k0 = tile_row[blockIdx.x];
    const uint32_t kn = tile_row[blockIdx.x + 1];
    const uint32_t klast = ((uint64_t)roff[kn] < tend) ? kn : kn - 1u;
    const uint32_t nrows = klast - k0 + 1u;
    const bool starts_before = (uint64_t)roff[k0] < tbeg;
    const bool ends_after = (uint64_t)roff[klast + 1] > tend;

    for (uint32_t j = threadIdx.x; j <= nrows; j += kTileThreads) {
        uint64_t o = (uint64_t)roff[k0 + j];
        o = o < tbeg ? tbeg : (o > tend ? tend : o);
        s_off[j] = (uint32_t)(o - tbeg);
        if (j < nrows) {
            s_acc1[j] = 0ull;
            s_acc2[j] = 0u;
        }
    }
    __syncthreads();

    const uint32_t a = threadIdx.x * kEdgesPerThread;
    if (a < tlen) {
        const uint32_t b = min(a + (uint32_t)kEdgesPerThread, tlen);
        const uint32_t cnt = b - a;
        uint32_t v[kEdgesPerThread];
        if (cnt == kEdgesPerThread) {
            const uint4* p = reinterpret_cast<const uint4*>(idx + tbeg + a);
            const uint4 q0 = __ldg(p), q1 = __ldg(p + 1);
            v[0] = q0.x; v[1] = q0.y; v[2] = q0.z; v[3] = q0.w;
            v[4] = q1.x; v[5] = q1.y; v[6] = q1.z; v[7] = q1.w;
        } else {
#pragma unroll
            for (int i = 0; i < kEdgesPerThread; ++i) v[i] = (uint32_t)i < cnt ? __ldg(idx + tbeg + a + i) : 0u;
        }
        uint32_t c[kEdgesPerThread];
#pragma unroll
        for (int i = 0; i < kEdgesPerThread; ++i) c[i] = (uint32_t)i < cnt ? __ldg(col + v[i]) : 0u;
        uint64_t w[kEdgesPerThread];
        if (WEIGHTED) {
#pragma unroll
            for (int i = 0; i < kEdgesPerThread; ++i) w[i] = (uint32_t)i < cnt ? __ldg(wt + tbeg + a + i) : 0ull;
        }

        // row containing arc a: largest j with s_off[j] <= a
        uint32_t lo = 0, hi = nrows - 1u;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (s_off[mid] <= a) lo = mid; else hi = mid - 1u;
        }
        uint32_t j = lo;
        uint64_t acc1 = 0;
        uint32_t acc2 = 0;
        auto flush = [&](uint32_t jj) {
            const bool sb = (jj == 0u) && starts_before;
            const bool ea = (jj == nrows - 1u) && ends_after;
            if (!sb && !ea && s_off[jj] >= a && s_off[jj + 1] <= b) {
                const uint32_t node = rows[k0 + jj];
                sig1[node] = acc1;
                sig2[node] = acc2;
            } else {
                atomicAdd(&s_acc1[jj], (unsigned long long)acc1);
                atomicAdd(&s_acc2[jj], acc2);
            }
        };
#pragma unroll
        for (int i = 0; i < kEdgesPerThread; ++i) {
            if ((uint32_t)i < cnt) {
                const uint32_t e = a + i;
                while (e >= s_off[j + 1]) {
                    flush(j);
                    acc1 = 0;
                    acc2 = 0;
                    ++j;
                }
                uint64_t t1 = fmix64((uint64_t)c[i] ^ salt1);
                uint32_t t2 = fmix32(c[i] ^ salt2);
                if (WEIGHTED) {
                    t1 *= w[i];
                    t2 *= (uint32_t)w[i];
                }
                acc1 += t1;
                acc2 += t2;
            }
        }
        flush(j);
    }
    __syncthreads();

    for (uint32_t jj = threadIdx.x; jj < nrows; jj += kTileThreads) {
        const bool sb = (jj == 0u) && starts_before;
        const bool ea = (jj == nrows - 1u) && ends_after;
        const uint32_t rs = s_off[jj], re = s_off[jj + 1];
        if (!sb && !ea && rs / kEdgesPerThread == (re - 1u) / kEdgesPerThread) continue;  // written by its thread
        const uint32_t node = rows[k0 + jj];
        if (!sb && !ea) {
            sig1[node] = s_acc1[jj];
            sig2[node] = s_acc2[jj];
        } else {
            atomicAdd(&sig1[node], s_acc1[jj]);
            atomicAdd(&sig2[node], s_acc2[jj]);
        }
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
