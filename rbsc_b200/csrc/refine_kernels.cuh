// refine_kernels.cuh -- the per-round kernels of the colour-refinement loop.
//
// One pass (reference: the body of the round loop, src/rbsc/rbsc.cu:354-425):
//   k_signature    sig(u) = sum over u's arcs of wt * H(colour(v))    (rbsc.cu:80-87 + ReduceByKey 366-382)
//   k_insert_list  (colour(u), sig(u)) -> relabel-table slot           (replaces the sorts + scan of 384-396)
//   k_relabel_list new colour = smallest member of the slot's class    (replaces reorder 396)
//   k_follow       arc-less nodes take their representative's colour
//   k_fixpoint     block count unchanged -> done                        (replaces the D2H + host test of 398-402, 425)
//   k_compact_*    drop what can no longer change (see below)
// The reference's injectivity loop (rbsc.cu:404-419) has no counterpart: the
// per-arc term here is a bijection of the colour by construction.
//
// Work that cannot change the partition is dropped as the refinement goes:
//   - a singleton block never splits again, so its node leaves the relabel
//     list and its row leaves the signature pass (the arc set is compacted on
//     the device whenever it shrank by a quarter);
//   - nodes without arcs that share an initial colour have the same
//     signature (0) in every pass, so they stay together for good: one
//     representative per such group goes through the relabel, the others
//     copy its colour.
// The colour array is updated in place: every pass reads the colours of the
// previous pass in k_signature / k_insert before k_relabel overwrites them.
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
    uint32_t rep_changed;    // a representative's colour changed in the running pass
    uint32_t count;          // blocks counted by the running pass
    uint32_t prev;           // blocks after the last completed pass
    uint32_t done;           // fixpoint reached
    uint32_t error;          // device error bits (kErr*)
    uint32_t max_rounds;
    uint32_t stamp;          // relabel-table stamp of the running pass, 1..255
    uint32_t clear_pending;  // table must be cleared before the running pass
    uint32_t hash_bits;      // test hook: signatures truncated to this many bits (0 = off)
    uint32_t handoff;        // the active set is small: the persistent kernel takes over
    uint32_t ranks;          // initial classes given a dense rank by k_insert_init
    uint32_t rank_bad;       // k_insert_init could not rank every class (dense ranks by scan instead)
    uint32_t active_nodes;   // listed nodes after the last compaction
    uint32_t active_rows;    // rows of the active arc set after the last compaction
    uint32_t active_arcs;    // its arcs (saturating at 2^32 - 1)
    uint32_t pad2;
    uint64_t seed;
    uint32_t pcount[2];      // k_refine_persistent: block counts of even / odd passes
    uint32_t prep[2];        // k_refine_persistent: rep_changed of even / odd passes
    uint32_t round_blocks[kRoundLog];
};

// The pass bodies read the pass number (and stamp) from RoundState unless the
// caller passes its own copy (the persistent kernel keeps them per block).
constexpr uint32_t kRoundFromState = 0xffffffffu;

constexpr uint32_t kErrProbe = 1u;   // relabel table full (cannot happen at load <= 1/2)
constexpr uint32_t kErrRounds = 2u;  // max_rounds reached
constexpr uint32_t kErrBarrier = 4u; // a grid barrier of the persistent kernel timed out
constexpr uint32_t kErrStage = 8u;   // a staged (bulk async) copy of k_signature_staged did not complete
constexpr uint32_t kErrInput = 16u;  // an uploaded head is >= N (k_validate_heads)

// Heads [a0, a1) of an upload that arrives during the first pass: any head
// >= n sets kErrInput, and the signature kernels that would gather it return
// without reading (they check the error word first).
static __global__ void k_validate_heads(uint64_t a0, uint64_t a1, uint32_t n, const uint32_t* __restrict__ idx,
                                        RoundState* __restrict__ st)
{
    bool bad = false;
    for (uint64_t k = a0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a1; k += (uint64_t)gridDim.x * blockDim.x)
        bad |= idx[k] >= n;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&st->error, kErrInput);
}

// What the pass kernels work on; the compaction kernels shrink it.
struct ActiveSet {
    // arc set of k_signature: non-empty rows, their arcs, the tiling
    const uint32_t* rows;      // node of each row (K)
    const void* roff;          // first arc of each row (K+1; uint64 when roff64, else uint32)
    const uint32_t* tile_row;  // row holding the first arc of each tile (ntiles+1)
    const uint8_t* head8;      // row-head bitmap
    const uint32_t* idx;       // arc heads
    const uint64_t* wt;        // arc weights or null
    const uint32_t* split;     // rows crossing a tile edge
    uint64_t m;
    uint32_t K;
    uint32_t ntiles;
    uint32_t nsplit;
    uint32_t roff64;
    // node list of the hash relabel: entries node | kRepFlag
    const uint32_t* nodes;
    uint32_t nnodes;
    uint32_t retired;          // singleton blocks dropped from the node list
    // compaction bookkeeping
    unsigned long long rowctr; // (rows << 32) | arcs reserved in the destination arc set
    uint32_t nodectr;          // entries written to the destination node list
    uint32_t splitctr;         // rows appended to the destination split list
    uint32_t do_copy;          // the arc set is rebuilt in this pass
    uint32_t new_K;
    uint32_t new_m;
    uint32_t dst_arcs;         // which compacted arc buffer the next rebuild writes
    uint32_t dst_nodes;        // which node-list buffer the next compaction writes
    uint32_t compact_arcs;     // arc-set compaction allowed
    uint32_t nfollow;          // follower list length
    uint64_t dst_cap;          // arcs the compaction buffers hold
    unsigned long long arcctr; // arcs of the kept rows, counted without the 32-bit limit of rowctr
};

// Per-node signature: the 64-bit and the 32-bit sum side by side in 16 B, so
// that one store or one load of a node's signature touches one 32-B sector
// (two separate arrays cost two scattered sectors per node).
struct __align__(16) Sig {
    unsigned long long s1;
    uint32_t s2;
    uint32_t pad;
};

__device__ __forceinline__ void sig_store(Sig* p, uint64_t s1, uint32_t s2)
{
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(s1, (unsigned long long)s2);
}

__device__ __forceinline__ void sig_add(Sig* p, uint64_t s1, uint32_t s2)
{
    atomicAdd(&p->s1, (unsigned long long)s1);
    atomicAdd(&p->s2, s2);
}

__device__ __forceinline__ void sig_load(const Sig* p, uint64_t& s1, uint32_t& s2)
{
    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
    s1 = v.x;
    s2 = (uint32_t)v.y;
}

// Node-list flag: the node represents a group of arc-less nodes with the same
// initial colour, so its block is never a singleton.
constexpr uint32_t kRepFlag = 0x80000000u;
constexpr int kListBuf = 2048;  // shared-memory buffer of the buffered list appends (BlockAppend)

// Static pointers of the ping-pong compaction buffers.
struct CompactBufs {
    uint32_t* rows[2];
    uint32_t* off[2];      // uint32 offsets (K+1)
    uint64_t* src[2];      // where each row's arcs start in the source arc set
    uint32_t* idx[2];
    uint64_t* wt[2];
    uint8_t* head8[2];
    uint32_t* tile_row[2];
    uint32_t* split[2];
    uint32_t* nodes[2];
    uint32_t* chunk_row[2];  // row holding the first arc of each 16-arc destination chunk
};

// Pass modes of the exact (non-hashed) relabels over all nodes.
constexpr int kModeInit = 1;    // key = initial colour
constexpr int kModeRepair = 2;  // key = (label, failed-exact-check flag)

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
// several nodes with this key, so the class is not a singleton.  Returns the
// slot; *claimed = this call created the class.
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
// The list passes' relabel table: 8-byte entries, half the bytes of Entry per
// probe (a 32-B sector holds four), cleared over the pass's window before its
// inserts (no stamp).  Entry word: low 32 bits = value (smallest member |
// kJoined), high 32 bits = tag (23 bits of the key's hash, top bit set so a
// claimed entry is never 0) << 8 | probe distance d.  A key is identified by
// its tag and its home slot (= slot - d): 23 + log2(window) bits of a 64-bit
// hash of (k1, k2), 47 bits for a 2^24-entry window.  Two different keys that
// share both would be merged into one class; the exact check at the fixpoint
// finds and splits any such merge, as it does for signature collisions.
// ---------------------------------------------------------------------------
constexpr uint32_t kProbeMax8 = 256;  // d fits in 8 bits

// load_first: read the entry before any atomic and try the claim only on an
// empty one.  A class that many nodes join (the first pass, whose keys are the
// few initial classes' refinements) then costs plain loads at its entry
// instead of an atomic per joining group, which serialise at one L2 slice;
// otherwise (most inserts claim a new class) the CAS goes first and saves the
// load's round trip.
__device__ __forceinline__ uint32_t table_insert8(unsigned long long* tab, uint32_t log2win, uint64_t k1, uint32_t k2,
                                                  uint32_t u, bool multi, bool* claimed, uint32_t* err, bool load_first)
{
    const uint64_t h = fmix64(k1 ^ ((uint64_t)(k2 & 0xffffff00u) * kGolden));
    const uint32_t mask = (1u << log2win) - 1u;
    const uint32_t tag = ((uint32_t)(h >> 8) & 0x7fffffu) | 0x800000u;
    uint32_t s = (uint32_t)(h >> (64 - log2win)) & mask;
    const uint32_t val = u | (multi ? kJoined : 0u);
    for (uint32_t d = 0; d < kProbeMax8 && d <= mask; ++d, s = (s + 1u) & mask) {
        const uint32_t hi = (tag << 8) | d;
        unsigned long long old = load_first ? *reinterpret_cast<volatile unsigned long long*>(tab + s) : 0ull;
        if (old == 0ull) {
            old = atomicCAS(tab + s, 0ull, ((unsigned long long)hi << 32) | val);
            if (old == 0ull) {
                *claimed = true;
                return s;
            }
        }
        if ((uint32_t)(old >> 32) == hi) {
            const uint32_t v = (uint32_t)old;
            if (!(v & kJoined) || (v & kLabelMask) > u) {
                uint32_t* vp = reinterpret_cast<uint32_t*>(tab + s);  // the value word (little-endian low half)
                atomicOr(vp, kJoined);
                atomicMin(vp, u | kJoined);
            }
            *claimed = false;
            return s;
        }
    }
    atomicOr(err, kErrProbe);
    *claimed = false;
    return 0;
}

// New colour word from an 8-byte entry (see relabel_one).
template <bool NC>
__device__ __forceinline__ uint32_t relabel_one8(uint32_t c, const unsigned long long* tab, uint32_t s)
{
    if (c & kSingleton) return c;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(tab + s);
    const uint32_t v = NC ? __ldg(w) : __ldcg(w);
    return (v & kLabelMask) | ((v & kJoined) ? 0u : kSingleton);
}

// ---------------------------------------------------------------------------
// Per-arc term of the signature: an injective function of the head's label
// (the multiply by an odd constant, the xor-shift and the second multiply are
// all bijections of uint64), salted per pass.  t1 feeds the 64-bit sum, t2 a
// second, independent-looking 32-bit sum.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void arc_terms(uint32_t c, uint64_t salt, uint64_t& t1, uint32_t& t2)
{
    uint64_t y = (uint64_t)((c & kLabelMask) ^ (uint32_t)salt) * 0x9e3779b97f4a7c15ull;
    y ^= y >> 32;
    y *= 0xd6e8feb86659fd93ull;
    y ^= y >> 32;
    t1 = y + (salt >> 32);
    t2 = (uint32_t)(y >> 32) * 0x2545f491u + (uint32_t)y * ((uint32_t)y | 1u);
}

// ---------------------------------------------------------------------------
// k_signature: edge-balanced tiles of 512 arcs, one tile at a time per warp
// (persistent warps).  Lane l owns the 16 consecutive arcs [16l, 16l+16) of
// the tile: four 16-byte loads of heads, two bytes of the row-head bitmap (bit
// j set = arc 16l+j starts a row), 16 gathered head colours.  A warp exclusive
// scan of the head counts gives every lane the index of its first row.  Each
// lane folds its arcs:
//   - rows that start and end inside its 16 arcs are written directly,
//   - the part before its first head belongs to the row continuing from the
//     previous lane, the part after its last head to the row continuing into
//     the next lane;
// a warp segmented scan joins the parts of rows that span lanes, and the lane
// in which such a row ends writes it.  A row that crosses a tile edge is added
// to global memory atomically (its signature was zeroed beforehand).  Sums
// are modulo 2^64 / 2^32, so the split into partial sums does not change the
// result.  Warps are independent: no shared memory, no block barrier.
// ---------------------------------------------------------------------------
// ColT: the gathered colour.  uint32_t = the colour word (label); the first
// pass may instead gather the dense rank of the initial class as uint8_t /
// uint16_t when there are few initial classes (a narrower array, mostly L1/L2
// resident).  Any injective relabelling of the colours gives the same
// partition.
// Colour gathers go through the read-only path (ld.global.nc) in the pass
// kernels, where the colours do not change during the launch; the persistent
// kernel rewrites them between its phases, so it reads them at L2 (NC false).
template <bool NC, typename ColT>
__device__ __forceinline__ uint32_t gather_col(const ColT* p)
{
    if constexpr (NC) return (uint32_t)__ldg(p);
    else return (uint32_t)__ldcg(p);
}

// Hot heads (first pass, 1-byte class ranks): a head with bit 31 set is the
// slot of one of the most pointed-to nodes, whose rank sits in shared memory
// (s_hot); any other head is a node id.  Node ids are < 2^31.
constexpr uint32_t kHotFlag = 0x80000000u;

template <bool NC, typename ColT, bool HOT>
__device__ __forceinline__ uint32_t gather_head(const ColT* col, const uint8_t* s_hot, uint32_t h)
{
    if constexpr (HOT) {
        if (h & kHotFlag) return (uint32_t)s_hot[h & ~kHotFlag];
    }
    return gather_col<NC>(col + h);
}

// A range of tiles [lo, hi) whose heads (and weights) were copied to a chunk
// buffer that starts at arc `base` (streamed arc sets); the default range is
// every tile, read from the active set's own arrays.
struct TileRange {
    uint32_t lo, hi;
    const uint32_t* idx;
    const uint64_t* wt;
    uint64_t base;
};

// The fold of one tile, once the lane has its head bits (hb, bit j = arc
// a + j starts a row), the colours c[] of its cnt heads and, weighted, their
// weights: per-lane partial sums, a warp segmented scan across lanes, the
// row signatures written (rows crossing a tile edge added atomically).
template <bool WEIGHTED>
__device__ __forceinline__ void signature_fold(uint32_t lane, uint32_t a, uint32_t cnt, uint32_t tlen, uint64_t tend, uint64_t m,
                                               uint32_t k0, uint32_t h0, uint32_t hb, const uint32_t (&c)[kEdgesPerThread],
                                               const uint64_t (&w)[kEdgesPerThread], uint64_t salt,
                                               const uint32_t* __restrict__ rows, const uint8_t* __restrict__ head8,
                                               Sig* __restrict__ sig)
{
    // row of arc a-1 (or of arc a when arc a does not start a row):
    // k0 + (heads in tile arcs [0, a)) - h0
    const uint32_t nheads = (uint32_t)__popc(hb);
    uint32_t hs = nheads;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, hs, d);
        if (lane >= (uint32_t)d) hs += o;
    }
    const uint32_t kbase = k0 + hs - nheads - h0;

    // fold: `pre` = arcs before this lane's first head, `cur` = the row
    // opened by the latest head; a row closed inside the lane is written
    uint64_t pre1 = 0, cur1 = 0;
    uint32_t pre2 = 0, cur2 = 0;
    uint32_t nh = 0;
    // running sums: a row's sum is the difference of the running sums at its
    // two ends (wrap-around arithmetic); every arc adds unconditionally
    uint64_t run1 = 0, last1 = 0;
    uint32_t run2 = 0, last2 = 0;
#pragma unroll
    for (int i = 0; i < kEdgesPerThread; ++i) {
        if ((uint32_t)i < cnt) {
            if ((hb >> i) & 1u) {
                if (nh > 0) {
                    const uint32_t node = rows[kbase + nh];
                    sig_store(&sig[node], run1 - last1, run2 - last2);
                } else {
                    pre1 = run1;
                    pre2 = run2;
                }
                last1 = run1;
                last2 = run2;
                ++nh;
            }
            uint64_t t1;
            uint32_t t2;
            arc_terms(c[i], salt, t1, t2);
            if (WEIGHTED) {
                t1 *= w[i];
                t2 *= (uint32_t)w[i];
            }
            run1 += t1;
            run2 += t2;
        }
    }
    if (nh == 0) {
        pre1 = run1;
        pre2 = run2;
    } else {
        cur1 = run1 - last1;
        cur2 = run2 - last2;
    }

    // warp inclusive segmented scan of the lanes' trailing parts (a
    // segment starts at every lane with a head)
    uint32_t f = nh > 0 ? 1u : 0u;
    uint64_t c1 = f ? cur1 : pre1;
    uint32_t c2 = f ? cur2 : pre2;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t fo = __shfl_up_sync(0xffffffffu, f, d);
        const uint64_t vo1 = __shfl_up_sync(0xffffffffu, c1, d);
        const uint32_t vo2 = __shfl_up_sync(0xffffffffu, c2, d);
        if (lane >= (uint32_t)d) {
            if (!f) {
                c1 += vo1;
                c2 += vo2;
            }
            f |= fo;
        }
    }
    uint64_t cin1 = __shfl_up_sync(0xffffffffu, c1, 1);
    uint32_t cin2 = __shfl_up_sync(0xffffffffu, c2, 1);
    if (lane == 0) {
        cin1 = 0;
        cin2 = 0;
    }
    if (cnt == 0) return;

    // the row continuing into this lane ends here when this lane has a head
    if (nh > 0 && (a > 0 || !(hb & 1u))) {
        const uint32_t node = rows[kbase];
        const uint64_t tot1 = cin1 + pre1;
        const uint32_t tot2 = cin2 + pre2;
        if (kbase == k0 && !h0) {  // began in an earlier tile
            sig_add(&sig[node], tot1, tot2);
        } else {
            sig_store(&sig[node], tot1, tot2);
        }
    }
    // the last lane of the tile closes the tile's last row
    if (a + cnt == tlen) {
        const uint32_t klast = kbase + nh;
        const bool ends = (tend == m) || (head8[tend >> 3] & 1u);
        const bool began_before = (klast == k0 && !h0);
        const uint32_t node = rows[klast];
        if (ends && !began_before) {
            sig_store(&sig[node], c1, c2);
        } else {
            sig_add(&sig[node], c1, c2);
        }
    }
}

// HOT: the heads come from hot_idx (same positions as the active set's
// heads, hot ones encoded as kHotFlag | slot) and ColT is the 1-byte rank.
// WPB: warps per block.
template <bool WEIGHTED, typename ColT, bool NC = true, bool RANGE = false, bool HOT = false,
          uint32_t WPB = kTileThreads / 32>
__device__ __forceinline__ void signature_body(const ActiveSet* __restrict__ as, const RoundState* __restrict__ st,
                                               const ColT* __restrict__ col, Sig* __restrict__ sig,
                                               TileRange rng = TileRange{0u, 0u, nullptr, nullptr, 0ull},
                                               const uint32_t* __restrict__ hot_idx = nullptr,
                                               const uint8_t* __restrict__ s_hot = nullptr,
                                               uint32_t round = kRoundFromState)
{
    static_assert(!HOT || (sizeof(ColT) == 1 && !RANGE), "hot heads: resident arcs, 1-byte ranks");
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ntiles = RANGE ? rng.hi : as->ntiles;
    const uint64_t m = as->m;
    const uint32_t* __restrict__ rows = as->rows;
    const uint32_t* __restrict__ tile_row = as->tile_row;
    const uint8_t* __restrict__ head8 = as->head8;
    // RANGE: idx[e - base] / wt[e - base] hold arc e of the chunk
    const uint32_t* __restrict__ idx = HOT ? hot_idx : (RANGE ? rng.idx : as->idx);
    const uint64_t* __restrict__ wt = RANGE ? rng.wt : as->wt;
    const uint64_t ebase = RANGE ? rng.base : 0ull;
    const uint64_t salt = pass_salt1(st->seed, round == kRoundFromState ? st->round : round);
    const uint32_t warps = gridDim.x * WPB;

    for (uint32_t tile = (RANGE ? rng.lo : 0u) + blockIdx.x * WPB + (threadIdx.x >> 5); tile < ntiles;
         tile += warps) {
        const uint64_t tbeg = (uint64_t)tile * kTileEdges;
        const uint32_t tlen = (uint32_t)min((uint64_t)kTileEdges, m - tbeg);
        const uint64_t tend = tbeg + tlen;
        const uint32_t k0 = tile_row[tile];
        const uint32_t h0 = head8[tbeg >> 3] & 1u;  // the tile's first arc starts a row
        const uint32_t a = lane * kEdgesPerThread;
        const uint32_t cnt = a < tlen ? min((uint32_t)kEdgesPerThread, tlen - a) : 0u;

        uint32_t hb = 0;
        uint32_t c[kEdgesPerThread];
        uint64_t w[kEdgesPerThread];
        static_assert(sizeof(ColT) <= 4, "colour type");
        if (cnt == kEdgesPerThread) {
            hb = *reinterpret_cast<const uint16_t*>(head8 + ((tbeg + a) >> 3));
            const uint4* p = reinterpret_cast<const uint4*>(idx + (tbeg - ebase) + a);
            const uint4 q0 = __ldcs(p), q1 = __ldcs(p + 1), q2 = __ldcs(p + 2), q3 = __ldcs(p + 3);
            c[0] = gather_head<NC, ColT, HOT>(col, s_hot, q0.x); c[1] = gather_head<NC, ColT, HOT>(col, s_hot, q0.y);
            c[2] = gather_head<NC, ColT, HOT>(col, s_hot, q0.z); c[3] = gather_head<NC, ColT, HOT>(col, s_hot, q0.w);
            c[4] = gather_head<NC, ColT, HOT>(col, s_hot, q1.x); c[5] = gather_head<NC, ColT, HOT>(col, s_hot, q1.y);
            c[6] = gather_head<NC, ColT, HOT>(col, s_hot, q1.z); c[7] = gather_head<NC, ColT, HOT>(col, s_hot, q1.w);
            c[8] = gather_head<NC, ColT, HOT>(col, s_hot, q2.x); c[9] = gather_head<NC, ColT, HOT>(col, s_hot, q2.y);
            c[10] = gather_head<NC, ColT, HOT>(col, s_hot, q2.z); c[11] = gather_head<NC, ColT, HOT>(col, s_hot, q2.w);
            c[12] = gather_head<NC, ColT, HOT>(col, s_hot, q3.x); c[13] = gather_head<NC, ColT, HOT>(col, s_hot, q3.y);
            c[14] = gather_head<NC, ColT, HOT>(col, s_hot, q3.z); c[15] = gather_head<NC, ColT, HOT>(col, s_hot, q3.w);
        } else {
            if (cnt) hb = (uint32_t)(*reinterpret_cast<const uint16_t*>(head8 + ((tbeg + a) >> 3))) & ((1u << cnt) - 1u);
#pragma unroll
            for (int i = 0; i < kEdgesPerThread; ++i)
                c[i] = (uint32_t)i < cnt ? gather_head<NC, ColT, HOT>(col, s_hot, __ldcs(idx + (tbeg - ebase) + a + i)) : 0u;
        }
        if (WEIGHTED) {
#pragma unroll
            for (int i = 0; i < kEdgesPerThread; ++i) w[i] = (uint32_t)i < cnt ? __ldcs(wt + (tbeg - ebase) + a + i) : 0ull;
        }

        signature_fold<WEIGHTED>(lane, a, cnt, tlen, tend, m, k0, h0, hb, c, w, salt, rows, head8, sig);
    }
}

template <bool WEIGHTED, typename ColT>
static __global__ void __launch_bounds__(kTileThreads) k_signature(const ActiveSet* __restrict__ as,
                                                                   const RoundState* __restrict__ st,
                                                                   const ColT* __restrict__ col,
                                                                   Sig* __restrict__ sig)
{
    signature_body<WEIGHTED, ColT>(as, st, col, sig);
}

// ---------------------------------------------------------------------------
// k_signature_staged: the same fold, with each warp's tiles staged in shared
// memory by the bulk copy engine (cp.async.bulk, completion counted on an
// mbarrier) two tiles deep: while the warp folds tile i, the heads and
// row-head bits of its next tile are already on their way.  The staged heads
// never pass through L1, which keeps L1 for the gathered colours.  Measured
// on R-MAT-24's first pass it is slower than the plain loads (1.13 vs 0.96
// ms: the pass is bound by the L2->L1 colour gathers, and the per-tile wait
// and lower occupancy -- 64 registers, 34 KB of shared memory a block -- cost
// more than the staged head stream saves), so it is an option
// (rbsc_opts.sig_kernel = 2) and an autotuner candidate, not the default.  Every
// array it reads is padded to whole tiles, so a tile's copy is 2 KB of heads
// (the last one rounded up to 16 B) and 64 B of head bits, 16-B aligned.
// Waits are bounded: a copy that does not complete sets kErrStage, the warp
// waits (bounded again) for its other copy in flight and stops.
// ---------------------------------------------------------------------------
constexpr int kStageWarps = kTileThreads / 32;
constexpr uint32_t kStageSpins = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kStageSpins; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

template <typename ColT>
static __global__ void __launch_bounds__(kTileThreads) k_signature_staged(const ActiveSet* __restrict__ as,
                                                                          RoundState* __restrict__ st,
                                                                          const ColT* __restrict__ col, Sig* __restrict__ sig,
                                                                          TileRange rng, int use_range)
{
    __shared__ __align__(128) uint32_t s_idx[kStageWarps][2][kTileEdges];
    __shared__ __align__(16) uint8_t s_hd[kStageWarps][2][kTileEdges / 8];
    __shared__ __align__(8) uint64_t s_bar[kStageWarps][2];
    if (*(const volatile uint32_t*)&st->error) return;
    const uint32_t lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t ntiles = use_range ? rng.hi : as->ntiles;
    const uint64_t m = as->m;
    const uint32_t* __restrict__ rows = as->rows;
    const uint32_t* __restrict__ tile_row = as->tile_row;
    const uint8_t* __restrict__ head8 = as->head8;
    const uint32_t* __restrict__ idx = use_range ? rng.idx : as->idx;
    const uint64_t ebase = use_range ? rng.base : 0ull;
    const uint64_t salt = pass_salt1(st->seed, st->round);
    const uint32_t warps = gridDim.x * kStageWarps;
    uint64_t* bar = s_bar[wi];
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    // lane 0 asks for tile t in buffer b
    auto issue = [&](uint32_t t, int b) {
        const uint64_t tb = (uint64_t)t * kTileEdges;
        const uint32_t tl = (uint32_t)min((uint64_t)kTileEdges, m - tb);
        const uint32_t bytes = (tl * 4u + 15u) & ~15u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[b], bytes + kTileEdges / 8);
        bulk_copy_g2s(s_idx[wi][b], idx + (tb - ebase), bytes, &bar[b]);
        bulk_copy_g2s(s_hd[wi][b], head8 + (tb >> 3), kTileEdges / 8, &bar[b]);
    };
    uint32_t tile = (use_range ? rng.lo : 0u) + blockIdx.x * kStageWarps + wi;
    // bit b of `phases`: the parity buffer b waits for next; bit b of
    // `inflight`: a copy into buffer b is issued and not yet waited for
    uint32_t phases = 0u, inflight = 0u;
    if (tile < ntiles) {
        if (lane == 0) issue(tile, 0);
        inflight = 1u;
    }
    bool failed = false;
    for (uint32_t i = 0; tile < ntiles; tile += warps, ++i) {
        const int b = (int)(i & 1u);
        const uint32_t next = tile + warps;
        if (next < ntiles) {
            if (lane == 0) issue(next, b ^ 1);
            inflight |= 1u << (b ^ 1);
        }
        const bool ok = mbar_wait_bounded(&bar[b], (phases >> b) & 1u);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicOr(&st->error, kErrStage);
            failed = true;
            break;
        }
        phases ^= 1u << b;
        inflight &= ~(1u << b);
        const uint64_t tbeg = (uint64_t)tile * kTileEdges;
        const uint32_t tlen = (uint32_t)min((uint64_t)kTileEdges, m - tbeg);
        const uint64_t tend = tbeg + tlen;
        const uint32_t k0 = tile_row[tile];
        const uint8_t* hd = s_hd[wi][b];
        const uint32_t h0 = hd[0] & 1u;
        const uint32_t a = lane * kEdgesPerThread;
        const uint32_t cnt = a < tlen ? min((uint32_t)kEdgesPerThread, tlen - a) : 0u;
        uint32_t hb = cnt ? (uint32_t)*reinterpret_cast<const uint16_t*>(hd + (a >> 3)) : 0u;
        if (cnt < (uint32_t)kEdgesPerThread) hb &= (1u << cnt) - 1u;
        uint32_t c[kEdgesPerThread];
        uint64_t w[kEdgesPerThread];
        if (cnt == kEdgesPerThread) {
            // the lane's four 16-B quarters, read in a lane-rotated order so
            // that eight lanes of a phase hit distinct banks
            const uint4* p = reinterpret_cast<const uint4*>(&s_idx[wi][b][a]);
            const uint32_t r = lane & 3u;
            const uint4 v0 = p[(0u + r) & 3u], v1 = p[(1u + r) & 3u], v2 = p[(2u + r) & 3u], v3 = p[(3u + r) & 3u];
            // quarter q was read by load (q - r) & 3
            const uint4 q0 = r == 0 ? v0 : r == 1 ? v3 : r == 2 ? v2 : v1;
            const uint4 q1 = r == 0 ? v1 : r == 1 ? v0 : r == 2 ? v3 : v2;
            const uint4 q2 = r == 0 ? v2 : r == 1 ? v1 : r == 2 ? v0 : v3;
            const uint4 q3 = r == 0 ? v3 : r == 1 ? v2 : r == 2 ? v1 : v0;
            c[0] = gather_col<true>(col + q0.x); c[1] = gather_col<true>(col + q0.y);
            c[2] = gather_col<true>(col + q0.z); c[3] = gather_col<true>(col + q0.w);
            c[4] = gather_col<true>(col + q1.x); c[5] = gather_col<true>(col + q1.y);
            c[6] = gather_col<true>(col + q1.z); c[7] = gather_col<true>(col + q1.w);
            c[8] = gather_col<true>(col + q2.x); c[9] = gather_col<true>(col + q2.y);
            c[10] = gather_col<true>(col + q2.z); c[11] = gather_col<true>(col + q2.w);
            c[12] = gather_col<true>(col + q3.x); c[13] = gather_col<true>(col + q3.y);
            c[14] = gather_col<true>(col + q3.z); c[15] = gather_col<true>(col + q3.w);
        } else {
#pragma unroll
            for (int j = 0; j < kEdgesPerThread; ++j) c[j] = (uint32_t)j < cnt ? gather_col<true>(col + s_idx[wi][b][a + j]) : 0u;
        }
        signature_fold<false>(lane, a, cnt, tlen, tend, m, k0, h0, hb, c, w, salt, rows, head8, sig);
        __syncwarp();
    }
    // copies still in flight (the loop stopped early): wait for them, bounded
    if (failed)
        for (int b = 0; b < 2; ++b)
            if ((inflight >> b) & 1u) mbar_wait_bounded(&bar[b], (phases >> b) & 1u);
}

// The same over the tiles of one streamed chunk (see TileRange).
template <bool WEIGHTED, typename ColT>
static __global__ void __launch_bounds__(kTileThreads) k_signature_chunk(const ActiveSet* __restrict__ as,
                                                                         const RoundState* __restrict__ st,
                                                                         const ColT* __restrict__ col,
                                                                         Sig* __restrict__ sig, TileRange rng)
{
    if (*(const volatile uint32_t*)&st->error) return;  // e.g. a bad head in this chunk
    signature_body<WEIGHTED, ColT, true, true>(as, st, col, sig, rng);
}

// First pass when every node starts in one block (the reference's default):
// every arc's term is the same, so a row's signature is its length (or its
// total weight) times that term, and no arc needs to be read.
template <bool WEIGHTED>
static __global__ void __launch_bounds__(kNodeThreads) k_signature_uniform(const ActiveSet* __restrict__ as,
                                                                           const RoundState* __restrict__ st,
                                                                           const uint64_t* __restrict__ off,
                                                                           const uint64_t* __restrict__ wt, uint32_t c0,
                                                                           Sig* __restrict__ sig)
{
    const uint32_t K = as->K;
    const uint32_t* __restrict__ rows = as->rows;
    uint64_t t1;
    uint32_t t2;
    arc_terms(c0, pass_salt1(st->seed, st->round), t1, t2);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const uint32_t u = rows[k];
        const uint64_t b = off[u], e = off[u + 1];
        uint64_t w = e - b;
        uint32_t w2 = (uint32_t)w;
        if (WEIGHTED) {
            w = 0;
            w2 = 0;
            for (uint64_t j = b; j < e; ++j) {
                w += wt[j];
                w2 += (uint32_t)wt[j];
            }
        }
        sig_store(&sig[u], w * t1, w2 * t2);
    }
}

// Dense ranks of the classes (labels in increasing order): flag[u] = u is the
// smallest node of its class.
static __global__ void k_class_heads(uint32_t n, const uint32_t* __restrict__ col, uint32_t* __restrict__ flag)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) flag[u] = (col[u] & kLabelMask) == u ? 1u : 0u;
}

template <typename ColT>
static __global__ void k_class_ranks(uint32_t n, const uint32_t* __restrict__ col, const uint32_t* __restrict__ rank,
                                     ColT* __restrict__ out)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) out[u] = (ColT)rank[col[u] & kLabelMask];
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
// Relabel through the table.  Each node of a warp builds its key, groups with
// equal keys of the warp (__match_any_sync), and one lane probes the table
// once for the group, offering the group's smallest node as the class label.
// Counts the classes it creates.
// ---------------------------------------------------------------------------
// log2 of the table window used for a list of `count` keys (load <= 1/2).
__device__ __forceinline__ uint32_t table_window(uint32_t count, uint32_t log2size)
{
    uint32_t w = 10;
    while (w < log2size && (1ull << w) < 2ull * count) ++w;
    return w;
}

__device__ __forceinline__ void insert_warp(bool need, uint32_t u, uint32_t slot_index, bool rep, uint64_t k1, uint32_t k2,
                                            uint32_t stamp, Entry* tab, uint32_t log2size, uint32_t* slot, uint32_t* err,
                                            bool& new_block)
{
    const int lane = threadIdx.x & 31;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    const unsigned rep_mask = __ballot_sync(0xffffffffu, need && rep);
    if (need) {
        const unsigned peers = __match_any_sync(need_mask, k1) & __match_any_sync(need_mask, k2);
        const int leader = __ffs(peers) - 1;
        // the list is not in node order: the group's label candidate is its minimum
        const uint32_t umin = __reduce_min_sync(peers, u);
        uint32_t s = 0;
        bool claimed = false;
        if (lane == leader)
            s = table_insert(tab, log2size, k1, k2, stamp, umin, __popc(peers) > 1 || (rep_mask & peers), &claimed, err);
        s = __shfl_sync(peers, s, leader);
        slot[slot_index] = s;
        new_block = (lane == leader) && claimed;
    }
}

// insert_warp on the 8-byte table of the list passes.
__device__ __forceinline__ void insert_warp8(bool need, uint32_t u, uint32_t slot_index, bool rep, uint64_t k1, uint32_t k2,
                                             unsigned long long* tab, uint32_t log2win, uint32_t* slot, uint32_t* err,
                                             bool load_first, bool& new_block)
{
    const int lane = threadIdx.x & 31;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    const unsigned rep_mask = __ballot_sync(0xffffffffu, need && rep);
    if (need) {
        const unsigned peers = __match_any_sync(need_mask, k1) & __match_any_sync(need_mask, k2);
        const int leader = __ffs(peers) - 1;
        const uint32_t umin = __reduce_min_sync(peers, u);
        uint32_t s = 0;
        bool claimed = false;
        if (lane == leader)
            s = table_insert8(tab, log2win, k1, k2, umin, __popc(peers) > 1 || (rep_mask & peers), &claimed, err, load_first);
        s = __shfl_sync(peers, s, leader);
        slot[slot_index] = s;
        new_block = (lane == leader) && claimed;
    }
}

// Zeroes the 8-byte list table over the window the next inserts of the pass
// use (table_window of the listed node count): grid-stride, 16 B per store.
__device__ __forceinline__ void clear_window8(const ActiveSet* __restrict__ as, unsigned long long* __restrict__ tab,
                                              uint32_t log2size)
{
    const uint64_t entries = 1ull << table_window(as->nnodes, log2size);
    ulonglong2* t2 = reinterpret_cast<ulonglong2*>(tab);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < entries / 2; i += (uint64_t)gridDim.x * blockDim.x)
        t2[i] = make_ulonglong2(0ull, 0ull);
}

static __global__ void k_clear_window8(const ActiveSet* __restrict__ as, unsigned long long* __restrict__ tab,
                                       uint32_t log2size)
{
    clear_window8(as, tab, log2size);
}

__device__ __forceinline__ void count_blocks(bool new_block, uint32_t* counter)
{
    const unsigned nb = __ballot_sync(0xffffffffu, new_block);
    if ((threadIdx.x & 31) == 0 && nb) atomicAdd(counter, (uint32_t)__popc(nb));
}

// Slot of a listed node that keeps its block's label: the block's
// representative r (its smallest node), or a node whose signature equals r's.
constexpr uint32_t kRepSlot = 0xffffffffu;
constexpr int kInsertU = 1;  // list entries per thread and iteration of the hashed insert (2 measured slower)

// Hashed pass over the node list (grid-stride by blocks); returns this
// thread's count of new blocks.
//
// Representative fast path: the class of node u is (label, signature); the
// block's representative r = label is its smallest node, so every node whose
// signature equals r's lands in r's class, whose smallest member -- the new
// label -- is r again.  Those nodes (and r itself) skip the relabel table:
// they keep their colour, and mark joined[r] (= the pass tag) so that r knows
// its class has another member.  Only the nodes that differ from their
// representative go through the table, keyed by (label, signature) as before.
// Late passes, where few blocks split, do almost no table work.
//
// TAB: the table the keys go to -- unsigned long long (the 8-byte list table,
// zeroed over the window before the pass) or Entry (the 16-byte stamped
// table, which needs no zeroing: the persistent tail kernel uses it, where a
// zeroing per pass would cost more than its few inserts).
template <typename TAB>
__device__ __forceinline__ uint32_t insert_list_body(const ActiveSet* __restrict__ as, RoundState* __restrict__ st,
                                                     const uint32_t* __restrict__ col,
                                                     const Sig* __restrict__ sig, TAB* __restrict__ tab,
                                                     uint32_t log2size, uint32_t* __restrict__ slot,
                                                     uint32_t* __restrict__ joined, uint32_t round = kRoundFromState,
                                                     uint32_t stamp_in = 0u, uint32_t prev_in = 0u)
{
    const uint32_t nn = as->nnodes;
    const uint32_t* __restrict__ nodes = as->nodes;
    const uint32_t stamp = round == kRoundFromState ? st->stamp : stamp_in;
    const uint32_t hb = st->hash_bits;
    const uint64_t seed = st->seed;
    const uint32_t stride = gridDim.x * kNodeThreads;
    // probe only the first 2^k entries, 2^k >= 2 * list length: the table of
    // a late pass with few active nodes stays in L2
    const uint32_t log2win = table_window(nn, log2size);
    const uint32_t tag = (round == kRoundFromState ? st->round : round) + 1u;
    // many listed nodes per block so far: most inserts join a few big classes
    const uint32_t prev = round == kRoundFromState ? st->prev : prev_in;
    const bool load_first = (uint64_t)nn > 8ull * prev;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t made = 0;
    // each warp takes kInsertU x 32 consecutive list entries per iteration and
    // issues their loads (colour, then both signatures) side by side, so the
    // dependent chains of kInsertU nodes per thread overlap
    for (uint32_t base = (blockIdx.x * kNodeThreads + (threadIdx.x & ~31u)) * kInsertU; base < nn; base += stride * kInsertU) {
        uint32_t idx[kInsertU], e[kInsertU], u[kInsertU], c[kInsertU];
        uint64_t s1[kInsertU], r1[kInsertU];
        uint32_t s2[kInsertU], r2[kInsertU];
#pragma unroll
        for (int j = 0; j < kInsertU; ++j) {
            idx[j] = base + 32u * j + lane;
            e[j] = idx[j] < nn ? nodes[idx[j]] : 0u;
            u[j] = e[j] & ~kRepFlag;
        }
#pragma unroll
        for (int j = 0; j < kInsertU; ++j) c[j] = idx[j] < nn ? col[u[j]] : kSingleton;
#pragma unroll
        for (int j = 0; j < kInsertU; ++j) {
            s1[j] = r1[j] = 0ull;
            s2[j] = r2[j] = 0u;
            if (!(c[j] & kSingleton)) {
                const uint32_t lab = c[j] & kLabelMask;
                sig_load(&sig[u[j]], s1[j], s2[j]);
                if (u[j] != lab) sig_load(&sig[lab], r1[j], r2[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kInsertU; ++j) {
            const bool active = idx[j] < nn;
            bool need = active && !(c[j] & kSingleton);
            bool is_rep = false;
            uint64_t k1 = 0;
            uint32_t k2 = stamp;
            if (need) {
                const uint32_t lab = c[j] & kLabelMask;
                uint64_t a1 = s1[j], b1 = r1[j];
                uint32_t a2 = s2[j], b2 = r2[j];
                if (hb) {  // test hook: truncated (or, from 64 bits on, no) signatures
                    a1 = (hb >= 64) ? 0ull : (a1 & ((1ull << hb) - 1ull));
                    b1 = (hb >= 64) ? 0ull : (b1 & ((1ull << hb) - 1ull));
                    a2 = b2 = 0;
                }
                bool keep = u[j] == lab;
                is_rep = keep;
                if (!keep) {
                    keep = b1 == a1 && b2 == a2;
                    if (keep && joined[lab] != tag) joined[lab] = tag;
                }
                if (keep) {
                    slot[idx[j]] = kRepSlot;
                    need = false;
                } else {
                    k1 = a1 ^ fmix64(((uint64_t)lab << 1 | 1ull) * kGolden ^ seed);
                    k2 = ((a2 ^ fmix32(lab * 0x9e3779b1u + (uint32_t)seed)) & 0xffffff00u) | stamp;
                }
            }
            // a singleton or a representative stands for a block of its own
            // so far; the others count only when they open a class
            bool nb = (active && (c[j] & kSingleton)) || is_rep;
            if constexpr (sizeof(TAB) == 8)
                insert_warp8(need, u[j], idx[j], (e[j] & kRepFlag) != 0, k1, k2, tab, log2win, slot, &st->error, load_first, nb);
            else
                insert_warp(need, u[j], idx[j], (e[j] & kRepFlag) != 0, k1, k2, stamp, tab, log2win, slot, &st->error, nb);
            made += nb ? 1u : 0u;
        }
    }
    return made;
}

static __global__ void __launch_bounds__(kNodeThreads) k_insert_list(const ActiveSet* __restrict__ as, RoundState* __restrict__ st,
                                                                     const uint32_t* __restrict__ col,
                                                                     const Sig* __restrict__ sig,
                                                                     unsigned long long* __restrict__ tab, uint32_t log2size,
                                                                     uint32_t* __restrict__ slot, uint32_t* __restrict__ joined)
{
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    const uint32_t made = insert_list_body<unsigned long long>(as, st, col, sig, tab, log2size, slot, joined);
    block_count<kNodeThreads>(made, &st->count, sm);
}

// Exact pass over all nodes: the repair of a failed exact check (kModeRepair,
// aux = failure flags; the key is (label, failed)) or initial colours
// (kModeInit, aux = colours; k_insert_init is the fast form).  Grid-stride,
// one count per block.
template <int MODE>
static __global__ void __launch_bounds__(kNodeThreads) k_insert_all(uint32_t n, RoundState* __restrict__ st,
                                                                    const uint32_t* __restrict__ col,
                                                                    const uint32_t* __restrict__ aux, Entry* __restrict__ tab,
                                                                    uint32_t log2size, uint32_t* __restrict__ slot)
{
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    const uint32_t stamp = st->stamp;
    uint32_t made = 0;
    for (uint32_t base = blockIdx.x * kNodeThreads; base < n; base += gridDim.x * kNodeThreads) {
        const uint32_t u = base + threadIdx.x;
        const bool active = u < n;
        const uint32_t c = active ? col[u] : kSingleton;
        const bool need = active && (MODE == kModeInit || !(c & kSingleton));
        uint64_t k1 = 0;
        if (need) k1 = (MODE == kModeInit) ? (uint64_t)aux[u] : ((uint64_t)(c & kLabelMask) | ((uint64_t)(aux[u] != 0u) << 32));
        bool nb = active && !need;
        insert_warp(need, u, u, false, k1, stamp, stamp, tab, log2size, slot, &st->error, nb);
        made += nb ? 1u : 0u;
    }
    block_count<kNodeThreads>(made, &st->count, sm);
}

// Initial pass (key = initial colour, the same keys and table as
// k_insert_all<kModeInit>).  The initial colours of a large graph usually
// take few values, and with one probe per warp group every warp of the grid
// would hit the same few table entries, one after another in L2.  Here each
// block takes a contiguous stretch of nodes and first combines its keys in a
// shared-memory table (smallest node and count per key), then makes one
// global insert per distinct key, then hands the global slots back to its
// nodes.  A key whose probe sequence in the shared table is full (many
// distinct keys) goes to the global table per warp group instead.
constexpr int kInitSlots = 1024;
constexpr int kInitProbes = 32;

__device__ __forceinline__ int init_probe(const unsigned long long* s_key, uint32_t key)
{
    uint32_t h = (key * 0x9e3779b1u) >> (32 - 10);
    for (int p = 0; p < kInitProbes; ++p, h = (h + 1) & (kInitSlots - 1)) {
        const unsigned long long k = s_key[h];
        if (k == (unsigned long long)key) return (int)h;
        if (k == ~0ull) return -1;
    }
    return -1;
}

//
// Every class that a block claims gets a dense rank (0, 1, ... in claiming
// order) in srank[slot]; the first signature pass gathers these ranks as
// 8- or 16-bit colours when there are few classes.  A class claimed on the
// per-warp path gets none (rank_bad is raised and the ranks come from a scan).
static __global__ void __launch_bounds__(kNodeThreads) k_insert_init(uint32_t n, uint32_t chunk, RoundState* __restrict__ st,
                                                                     const uint32_t* __restrict__ init,
                                                                     Entry* __restrict__ tab, uint32_t log2size,
                                                                     uint32_t* __restrict__ slot, uint32_t* __restrict__ srank)
{
    static_assert(kInitSlots == 1024, "init_probe hashes to 10 bits");
    __shared__ unsigned long long s_key[kInitSlots];
    __shared__ uint32_t s_min[kInitSlots], s_cnt[kInitSlots], s_slot[kInitSlots];
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    constexpr unsigned long long kEmpty = ~0ull;
    for (int i = threadIdx.x; i < kInitSlots; i += kNodeThreads) {
        s_key[i] = kEmpty;
        s_min[i] = 0xffffffffu;
        s_cnt[i] = 0u;
    }
    __syncthreads();
    const uint32_t beg = blockIdx.x * chunk;
    const uint32_t end = (uint32_t)min((uint64_t)n, (uint64_t)beg + chunk);
    const uint32_t stamp = st->stamp;
    const int lane = threadIdx.x & 31;
    uint32_t made = 0;
    for (uint32_t base = beg; base < end; base += kNodeThreads) {
        const uint32_t u = base + threadIdx.x;
        const bool active = u < end;
        const uint32_t key = active ? init[u] : 0u;
        const unsigned am = __ballot_sync(0xffffffffu, active);
        bool overflow = false;
        if (active) {
            const unsigned peers = __match_any_sync(am, key);
            const int leader = __ffs(peers) - 1;
            const uint32_t umin = __reduce_min_sync(peers, u);
            int pos = -1;
            if (lane == leader) {
                uint32_t h = (key * 0x9e3779b1u) >> (32 - 10);
                for (int p = 0; p < kInitProbes; ++p, h = (h + 1) & (kInitSlots - 1)) {
                    const unsigned long long prev = atomicCAS(&s_key[h], kEmpty, (unsigned long long)key);
                    if (prev == kEmpty || prev == (unsigned long long)key) {
                        atomicMin(&s_min[h], umin);
                        atomicAdd(&s_cnt[h], (uint32_t)__popc(peers));
                        pos = (int)h;
                        break;
                    }
                }
            }
            pos = __shfl_sync(peers, pos, leader);
            overflow = pos < 0;
        }
        if (__any_sync(0xffffffffu, overflow)) {
            bool nb = false;
            insert_warp(overflow, u, u, false, (uint64_t)key, stamp, stamp, tab, log2size, slot, &st->error, nb);
            made += nb ? 1u : 0u;
            if (nb) st->rank_bad = 1u;
        }
    }
    __syncthreads();
    constexpr int kPer = kInitSlots / kNodeThreads;
    uint32_t claims = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * kNodeThreads;
        const unsigned long long k = s_key[i];
        bool claimed = false;
        if (k != kEmpty) s_slot[i] = table_insert(tab, log2size, k, stamp, stamp, s_min[i], s_cnt[i] > 1u, &claimed, &st->error);
        s_cnt[i] = claimed ? 1u : 0u;  // s_cnt is free from here on: the claimed flags
        claims += claimed ? 1u : 0u;
    }
    made += claims;
    uint32_t r0 = block_reserve_n<kNodeThreads>(claims, &st->ranks, sm);
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * kNodeThreads;
        if (s_cnt[i]) srank[s_slot[i]] = r0++;
    }
    __syncthreads();
    for (uint32_t base = beg; base < end; base += kNodeThreads) {
        const uint32_t u = base + threadIdx.x;
        if (u < end) {
            const int pos = init_probe(s_key, init[u]);
            if (pos >= 0) slot[u] = s_slot[pos];
        }
    }
    block_count<kNodeThreads>(made, &st->count, sm);
}

// New colour word from the table entry of the node's class.  The relabel
// kernels run after the inserts of their pass completed (an earlier launch),
// so they may read the table through the read-only path (NC), where the few
// entries of big classes stay in L1; the persistent kernel inserts and
// relabels in one launch and reads at L2.
template <bool NC>
__device__ __forceinline__ uint32_t relabel_one(uint32_t c, const Entry* tab, uint32_t s)
{
    if (c & kSingleton) return c;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(tab + s) + 3;
    const uint32_t v = NC ? __ldg(w) : __ldcg(w);
    return (v & kLabelMask) | ((v & kJoined) ? 0u : kSingleton);
}

// New colours of the node list, in place (slots are indexed by list
// position); also zeroes the signatures of the rows that cross a tile edge
// (the next pass adds into them atomically).  Four list entries per thread
// and iteration, so their dependent loads overlap.
template <bool NC, typename TAB>
__device__ __forceinline__ void relabel_list_body(const ActiveSet* __restrict__ as, RoundState* __restrict__ st,
                                                  uint32_t* __restrict__ col, const TAB* __restrict__ tab,
                                                  const uint32_t* __restrict__ slot, Sig* __restrict__ sig,
                                                  const uint32_t* __restrict__ joined, uint32_t round = kRoundFromState,
                                                  uint32_t* __restrict__ rep_changed = nullptr)
{
    const uint32_t tag = (round == kRoundFromState ? st->round : round) + 1u;
    uint32_t* const repc = rep_changed ? rep_changed : &st->rep_changed;
    const uint32_t nn = as->nnodes;
    const uint32_t* __restrict__ nodes = as->nodes;
    const uint32_t stride = gridDim.x * kNodeThreads;
    constexpr int U = 4;
    for (uint32_t i0 = blockIdx.x * kNodeThreads + threadIdx.x; i0 < nn; i0 += U * stride) {
        uint32_t u[U], s[U], c[U];
        bool rep[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t i = i0 + j * stride;
            const uint32_t e = i < nn ? nodes[i] : 0xffffffffu;
            u[j] = e == 0xffffffffu ? e : (e & ~kRepFlag);
            rep[j] = e != 0xffffffffu && (e & kRepFlag);
            s[j] = i < nn ? slot[i] : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) c[j] = u[j] != 0xffffffffu ? col[u[j]] : kSingleton;
        // most colours of a late pass do not change: no store (a partial
        // sector write) for those; a changed representative makes k_follow
        // run in this pass
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (u[j] == 0xffffffffu) continue;
            uint32_t nc = c[j];
            if (s[j] == kRepSlot) {
                // kept its block's label; the representative of a class that
                // nobody joined (and that stands for no follower) is alone
                if (!(c[j] & kSingleton) && (c[j] & kLabelMask) == u[j] && !rep[j] &&
                    (NC ? __ldg(joined + u[j]) : __ldcg(joined + u[j])) != tag)
                    nc = c[j] | kSingleton;
            } else {
                if constexpr (sizeof(TAB) == 8) nc = relabel_one8<NC>(c[j], tab, s[j]);
                else nc = relabel_one<NC>(c[j], tab, s[j]);
            }
            if (nc != c[j]) {
                col[u[j]] = nc;
                if (rep[j]) *repc = 1u;
            }
        }
    }
    const uint32_t ns = as->nsplit;
    const uint32_t* __restrict__ split = as->split;
    for (uint32_t i = blockIdx.x * kNodeThreads + threadIdx.x; i < ns; i += stride) {
        const uint32_t node = split[i];
        sig_store(&sig[node], 0ull, 0u);
    }
}

static __global__ void __launch_bounds__(kNodeThreads) k_relabel_list(const ActiveSet* __restrict__ as,
                                                                      RoundState* __restrict__ st, uint32_t* __restrict__ col,
                                                                      const unsigned long long* __restrict__ tab,
                                                                      const uint32_t* __restrict__ slot,
                                                                      Sig* __restrict__ sig, const uint32_t* __restrict__ joined)
{
    relabel_list_body<true, unsigned long long>(as, st, col, tab, slot, sig, joined);
}

// New colours of all nodes (after k_insert_all), in place.
// Initial pass (initlab non-null): every node is relabelled (col is not read)
// and its label is also written to initlab; with at most 65536 classes, all
// ranked by k_insert_init, the class rank goes to rank (8 or 16 bits).
static __global__ void __launch_bounds__(kNodeThreads) k_relabel_all(uint32_t n, uint32_t* __restrict__ col,
                                                                     const Entry* __restrict__ tab,
                                                                     const uint32_t* __restrict__ slot,
                                                                     uint32_t* __restrict__ initlab,
                                                                     const RoundState* __restrict__ st = nullptr,
                                                                     const uint32_t* __restrict__ srank = nullptr,
                                                                     void* __restrict__ rank = nullptr)
{
    const uint32_t classes = st ? st->count : 0xffffffffu;
    const int rank_bytes = (!st || st->rank_bad || classes > 65536u) ? 0 : (classes <= 256u ? 1 : 2);
    for (uint32_t u = blockIdx.x * kNodeThreads + threadIdx.x; u < n; u += gridDim.x * kNodeThreads) {
        uint32_t c = initlab ? 0u : col[u];
        if (!(c & kSingleton)) {
            const uint32_t s = slot[u];
            c = relabel_one<true>(c, tab, s);
            col[u] = c;
            if (rank_bytes == 1) static_cast<uint8_t*>(rank)[u] = (uint8_t)__ldg(srank + s);
            else if (rank_bytes == 2) static_cast<uint16_t*>(rank)[u] = (uint16_t)__ldg(srank + s);
        }
        if (initlab) initlab[u] = c & kLabelMask;
    }
}

// Followers (arc-less nodes that are not their group's representative) take
// the representative's colour.  pairs[i] = (follower, representative).
__device__ __forceinline__ void follow_body(const ActiveSet* __restrict__ as, const RoundState* __restrict__ st,
                                            const uint2* __restrict__ pairs, uint32_t* __restrict__ col,
                                            const uint32_t* rep_changed = nullptr)
{
    // the representatives' colours are those of their groups: they change
    // in the pass after the lists are built, and then only when a block of
    // arc-less nodes loses a member with arcs that merged into it by a hash
    // collision; nothing to copy otherwise
    if (!*(const volatile uint32_t*)(rep_changed ? rep_changed : &st->rep_changed)) return;
    const uint32_t nf = as->nfollow;
    const uint32_t stride = gridDim.x * kNodeThreads;
    for (uint32_t i = blockIdx.x * kNodeThreads + threadIdx.x; i < nf; i += stride) {
        const uint2 p = pairs[i];
        col[p.x] = col[p.y];
    }
}

static __global__ void __launch_bounds__(kNodeThreads) k_follow(const ActiveSet* __restrict__ as,
                                                                const RoundState* __restrict__ st,
                                                                const uint2* __restrict__ pairs, uint32_t* __restrict__ col)
{
    follow_body(as, st, pairs, col);
}

// k_fixpoint: one thread.  Closes the running pass and decides whether the
// device-side while loop runs another one.
//   hashed pass: blocks = classes found in the node list + retired singletons
//   (add_retired) or the count written by the sort-based relabel
//   init / repair pass: blocks = classes found over all nodes
constexpr int kFixHash = 0;
constexpr int kFixInit = 1;
constexpr int kFixRepair = 2;
template <int MODE>
__device__ __forceinline__ void fixpoint_body(RoundState* st, const ActiveSet* as, int add_retired)
{
    uint32_t cnt = st->count;
    st->count = 0;
    st->rep_changed = 0u;
    if (MODE == kFixHash) {
        if (add_retired) cnt += as->retired;
        const uint32_t r = st->round + 1u;
        st->round = r;
        if (r < kRoundLog) st->round_blocks[r] = cnt;
        if (cnt == st->prev) st->done = 1u;
    } else if (MODE == kFixInit) {
        st->round_blocks[0] = cnt;
        st->done = 0u;
        st->handoff = 0u;
    } else {
        st->done = 0u;
        st->handoff = 0u;
    }
    st->prev = cnt;
    const uint32_t stamp = st->stamp % 255u + 1u;
    st->stamp = stamp;
    st->clear_pending = stamp == 1u;
    if (!st->done && st->round >= st->max_rounds) st->error |= kErrRounds;
}

template <int MODE>
static __global__ void k_fixpoint(RoundState* st, const ActiveSet* as, int add_retired)
{
    fixpoint_body<MODE>(st, as, add_retired);
}

// ---------------------------------------------------------------------------
// Compaction (runs after k_fixpoint while the loop goes on).
// ---------------------------------------------------------------------------

// Keeps the non-singleton entries of the node list (order is not kept: the
// relabel does not depend on it); dropped nodes are singleton blocks for good.
// Appends are buffered per block (BlockAppend: one reservation per kListBuf
// kept nodes).  Warp-private buffers were measured slower here: the kept list
// is long, and one reservation per 256 entries on the single counter
// serialises in L2 (R-MAT-22 pass 1: 16.9 -> 26.0 us).
static __global__ void __launch_bounds__(kNodeThreads) k_compact_nodes(ActiveSet* __restrict__ as, const RoundState* __restrict__ st,
                                                                       const uint32_t* __restrict__ col, CompactBufs bufs)
{
    __shared__ BlockAppend<uint32_t, kListBuf, kNodeThreads> sa;
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    if (st->done || st->error) return;
    const uint32_t nn = as->nnodes;
    const uint32_t* __restrict__ src = as->nodes;
    uint32_t* __restrict__ dst = bufs.nodes[as->dst_nodes];
    const uint32_t stride = gridDim.x * kNodeThreads;
    uint32_t dropped = 0;
    block_append_begin(sa);
    for (uint32_t base = blockIdx.x * kNodeThreads; base < nn; base += stride) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < nn;
        const uint32_t e = valid ? src[i] : 0u;
        const bool keep = valid && !(col[e & ~kRepFlag] & kSingleton);
        block_append(sa, keep, e, &as->nodectr, dst);
        dropped += (valid && !keep) ? 1u : 0u;
    }
    block_append_flush(sa, &as->nodectr, dst);
    block_count<kNodeThreads>(dropped, &as->retired, sm);
}

// Counts and places the rows of non-singleton nodes of the current arc set in
// the destination arc set.  A block iteration takes kCompactRows x 256
// consecutive rows (row base + j*256 + thread, so every load is coalesced);
// one 64-bit atomic per iteration reserves (rows, arcs) together for the
// block, so row order and arc order agree in the destination (a counter that
// every block hits once per 256 rows serialises in L2).  Positions inside the
// iteration follow the source order (j, then warp, then lane), so the kept
// rows of one warp and item are written side by side.  The packed arcs are
// exact while the kept arcs stay below 2^32, which arcctr (64-bit) tells
// k_compact_decide; beyond that the positions are unused, and a row position
// past the current set's row count is not written.
constexpr int kCompactRows = 8;

static __global__ void __launch_bounds__(kNodeThreads, 4) k_compact_rows(ActiveSet* __restrict__ as, const RoundState* __restrict__ st,
                                                                      const uint32_t* __restrict__ col, CompactBufs bufs)
{
    constexpr int W = kNodeThreads / 32;
    __shared__ unsigned long long s_pre[kCompactRows][W];  // per (item, warp): packed total, then its exclusive offset
    __shared__ unsigned long long s_arcs[W];
    __shared__ unsigned long long s_base;
    if (st->done || st->error || !as->compact_arcs) return;
    const uint32_t K = as->K;
    const uint32_t* __restrict__ rows = as->rows;
    const bool r64 = as->roff64 != 0;
    const uint64_t* __restrict__ roff64 = reinterpret_cast<const uint64_t*>(as->roff);
    const uint32_t* __restrict__ roff32 = reinterpret_cast<const uint32_t*>(as->roff);
    const uint32_t d = as->dst_arcs;
    const uint64_t dst_cap = as->dst_cap;
    uint32_t* __restrict__ drows = bufs.rows[d];
    uint32_t* __restrict__ doff = bufs.off[d];
    uint64_t* __restrict__ dsrc = bufs.src[d];
    uint32_t* __restrict__ chunk_row = bufs.chunk_row[d];
    const uint64_t span = (uint64_t)kNodeThreads * kCompactRows;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t base = (uint64_t)blockIdx.x * span; base < K; base += (uint64_t)gridDim.x * span) {
        // every row of an arc set has at least one arc: deg 0 = not kept
        uint32_t node[kCompactRows], deg[kCompactRows];
        uint64_t start[kCompactRows];
        unsigned long long incl[kCompactRows];
#pragma unroll
        for (int j = 0; j < kCompactRows; ++j) {
            const uint64_t k = base + (uint64_t)j * kNodeThreads + threadIdx.x;
            node[j] = 0u;
            deg[j] = 0u;
            start[j] = 0ull;
            if (k < K) node[j] = rows[k];
        }
#pragma unroll
        for (int j = 0; j < kCompactRows; ++j) {
            const uint64_t k = base + (uint64_t)j * kNodeThreads + threadIdx.x;
            if (k < K && !(col[node[j]] & kSingleton)) {
                const uint64_t b = r64 ? roff64[k] : roff32[k];
                const uint64_t e = r64 ? roff64[k + 1] : roff32[k + 1];
                start[j] = b;
                deg[j] = (uint32_t)(e - b);
            }
        }
        unsigned long long arcs = 0;
#pragma unroll
        for (int j = 0; j < kCompactRows; ++j) {
            const unsigned long long v = deg[j] ? ((1ull << 32) | deg[j]) : 0ull;
            unsigned long long x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            incl[j] = x;
            if (lane == 31) s_pre[j][warp] = x;
            arcs += deg[j];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) arcs += __shfl_xor_sync(0xffffffffu, arcs, o);
        if (lane == 0) s_arcs[warp] = arcs;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long run = 0, run_arcs = 0;
            for (int j = 0; j < kCompactRows; ++j)
                for (int w = 0; w < W; ++w) {
                    const unsigned long long c = s_pre[j][w];
                    s_pre[j][w] = run;
                    run += c;
                }
            for (int w = 0; w < W; ++w) run_arcs += s_arcs[w];
            s_base = run ? atomicAdd(&as->rowctr, run) : 0ull;
            if (run_arcs) atomicAdd(&as->arcctr, run_arcs);
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kCompactRows; ++j) {
            if (!deg[j]) continue;
            const unsigned long long pos = s_base + s_pre[j][warp] + incl[j] - ((1ull << 32) | deg[j]);
            const uint32_t kn = (uint32_t)(pos >> 32);
            const uint32_t p0 = (uint32_t)pos;
            if (kn < K) {
                drows[kn] = node[j];
                doff[kn] = p0;
                dsrc[kn] = start[j];
                // the 16-arc destination chunks that start in this row
                // (within the buffers: past the capacity nothing is copied)
                if ((uint64_t)p0 + deg[j] <= dst_cap)
                    for (uint32_t c = (p0 + 15u) >> 4; (c << 4) < p0 + deg[j]; ++c) chunk_row[c] = kn;
            }
        }
        __syncthreads();
    }
}

// Decides whether the arc set is rebuilt: when its arcs dropped to 3/4 or less.
static __global__ void k_compact_decide(ActiveSet* as, const RoundState* st, CompactBufs bufs)
{
    if (st->done || st->error || !as->compact_arcs) {
        as->do_copy = 0;
        return;
    }
    // copy when the kept arcs fit the 32-bit destination offsets and the
    // compaction buffers, and dropped to 3/4 of the current set or less
    const uint64_t arcs = as->arcctr;
    const uint32_t nk = (uint32_t)(as->rowctr >> 32);
    const uint32_t nm = (uint32_t)arcs;
    const bool copy = nk > 0 && arcs < (1ull << 32) && arcs <= as->dst_cap && arcs * 4ull <= as->m * 3ull;
    as->do_copy = copy ? 1u : 0u;
    as->new_K = nk;
    as->new_m = nm;
    if (copy) {
        const uint32_t d = as->dst_arcs;
        bufs.off[d][nk] = nm;
        bufs.tile_row[d][(nm + kTileEdges - 1) / kTileEdges] = nk;
    }
}

// Copies the arcs of the kept rows (16 destination arcs per thread), and
// builds the destination's row-head bitmap, tile rows and split list.  A row
// entering the split list gets its signatures zeroed here.  COPY false: the
// bookkeeping only (the arcs were copied by k_compact_copy_tiles).
template <bool COPY>
static __global__ void __launch_bounds__(kNodeThreads, 4) k_compact_arcs(ActiveSet* __restrict__ as, CompactBufs bufs,
                                                                      Sig* __restrict__ sig)
{
    if (!as->do_copy) return;
    const uint32_t nk = as->new_K;
    const uint32_t nm = as->new_m;
    const uint32_t d = as->dst_arcs;
    const uint32_t* __restrict__ doff = bufs.off[d];
    const uint64_t* __restrict__ dsrc = bufs.src[d];
    const uint32_t* __restrict__ drows = bufs.rows[d];
    uint32_t* __restrict__ didx = bufs.idx[d];
    uint64_t* __restrict__ dwt = bufs.wt[d];
    const uint32_t* __restrict__ sidx = as->idx;
    const uint64_t* __restrict__ swt = as->wt;
    const uint32_t chunks = (nm + 15u) / 16u;
    const uint32_t stride = gridDim.x * kNodeThreads;
    const uint32_t* __restrict__ chunk_row = bufs.chunk_row[d];
    for (uint32_t ch = blockIdx.x * kNodeThreads + threadIdx.x; ch < chunks; ch += stride) {
        const uint32_t e0 = ch * 16u;
        const uint32_t cnt = min(16u, nm - e0);
        // row holding arc e0 (recorded by k_compact_rows); the row walk finds
        // each arc's source position first, so the 16 source loads below are
        // independent of one another
        const uint32_t k0 = chunk_row[ch];
        uint32_t k = k0;
        uint32_t rb = doff[k], re = doff[k + 1];
        uint64_t src = dsrc[k];
        uint32_t bits = 0;
        uint64_t from[16];
#pragma unroll
        for (uint32_t i = 0; i < 16u; ++i) {
            const uint32_t e = e0 + i;
            from[i] = 0ull;
            if (i < cnt) {
                while (e >= re) {
                    ++k;
                    rb = re;
                    re = doff[k + 1];
                    src = dsrc[k];
                }
                if (e == rb) bits |= 1u << i;
                from[i] = src + (e - rb);
            }
        }
        if (COPY) {
            uint32_t h[16];
#pragma unroll
            for (uint32_t i = 0; i < 16u; ++i) h[i] = i < cnt ? sidx[from[i]] : 0u;
            if (cnt == 16u) {
                uint4* q = reinterpret_cast<uint4*>(didx + e0);
                q[0] = make_uint4(h[0], h[1], h[2], h[3]);
                q[1] = make_uint4(h[4], h[5], h[6], h[7]);
                q[2] = make_uint4(h[8], h[9], h[10], h[11]);
                q[3] = make_uint4(h[12], h[13], h[14], h[15]);
            } else {
#pragma unroll
                for (uint32_t i = 0; i < 16u; ++i)
                    if (i < cnt) didx[e0 + i] = h[i];
            }
            if (swt) {
#pragma unroll
                for (uint32_t i = 0; i < 16u; ++i)
                    if (i < cnt) dwt[e0 + i] = swt[from[i]];
            }
        }
        *reinterpret_cast<uint16_t*>(bufs.head8[d] + (e0 >> 3)) = (uint16_t)bits;
        if ((e0 & (kTileEdges - 1u)) == 0u) {
            bufs.tile_row[d][e0 / kTileEdges] = k0;
            if (e0 > 0 && doff[k0] < e0) {  // row k0 crosses this tile edge
                const uint32_t node = drows[k0];
                const uint32_t p = atomicAdd(&as->splitctr, 1u);
                bufs.split[d][p] = node;
                sig_store(&sig[node], 0ull, 0u);
            }
        }
    }
}

// The copy of k_compact_arcs for a source arc set in host memory (read over
// the host link): one warp per 512-arc destination tile, lane l copying arcs
// l, l+32, ... so that each load of the warp reads 32 consecutive arcs of one
// row (one request) instead of 32 scattered ones.
static __global__ void __launch_bounds__(kNodeThreads) k_compact_copy_tiles(const ActiveSet* __restrict__ as, CompactBufs bufs)
{
    if (!as->do_copy) return;
    const uint32_t nk = as->new_K;
    const uint32_t nm = as->new_m;
    const uint32_t d = as->dst_arcs;
    const uint32_t* __restrict__ doff = bufs.off[d];
    const uint64_t* __restrict__ dsrc = bufs.src[d];
    uint32_t* __restrict__ didx = bufs.idx[d];
    uint64_t* __restrict__ dwt = bufs.wt[d];
    const uint32_t* __restrict__ sidx = as->idx;
    const uint64_t* __restrict__ swt = as->wt;
    const uint32_t* __restrict__ chunk_row = bufs.chunk_row[d];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tiles = (nm + kTileEdges - 1u) / kTileEdges;
    const uint32_t warps = gridDim.x * (kNodeThreads / 32);
    (void)nk;
    for (uint32_t t = blockIdx.x * (kNodeThreads / 32) + (threadIdx.x >> 5); t < tiles; t += warps) {
        const uint32_t e0 = t * kTileEdges + lane;
        if (e0 >= nm) continue;
        // from the row of e0's 16-arc chunk, at most 15 arcs ahead
        uint32_t k = chunk_row[e0 >> 4], rb = doff[k], re = doff[k + 1];
        while (e0 >= re) {
            ++k;
            rb = re;
            re = doff[k + 1];
        }
        uint64_t src = dsrc[k];
        uint32_t v[kTileEdges / 32];
        uint64_t w[kTileEdges / 32];
#pragma unroll
        for (uint32_t i = 0; i < kTileEdges / 32; ++i) {
            const uint32_t e = e0 + 32u * i;
            if (e < nm) {
                while (e >= re) {
                    ++k;
                    rb = re;
                    re = doff[k + 1];
                    src = dsrc[k];
                }
                v[i] = sidx[src + (e - rb)];
                if (swt) w[i] = swt[src + (e - rb)];
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < kTileEdges / 32; ++i) {
            const uint32_t e = e0 + 32u * i;
            if (e < nm) {
                didx[e] = v[i];
                if (swt) dwt[e] = w[i];
            }
        }
    }
}

// Switches the pass kernels to the compacted node list / arc set, and
// decides whether the device-side while loop runs another pass: not when the
// fixpoint is reached, an error was raised, or (handoff_arcs > 0) the active
// set became small enough for the persistent kernel, which then takes over.
static __global__ void k_compact_finalize(ActiveSet* as, RoundState* st, CompactBufs bufs, uint64_t handoff_arcs,
                                          uint32_t handoff_nodes, cudaGraphConditionalHandle handle, int use_handle)
{
    if (st->done || st->error) {
        if (use_handle) cudaGraphSetConditional(handle, 0u);
        return;
    }
    const uint32_t dn = as->dst_nodes;
    as->nodes = bufs.nodes[dn];
    as->nnodes = as->nodectr;
    as->nodectr = 0;
    as->dst_nodes = dn ^ 1u;
    if (as->do_copy) {
        const uint32_t d = as->dst_arcs;
        as->rows = bufs.rows[d];
        as->roff = bufs.off[d];
        as->roff64 = 0;
        as->tile_row = bufs.tile_row[d];
        as->head8 = bufs.head8[d];
        as->idx = bufs.idx[d];
        as->wt = as->wt ? bufs.wt[d] : nullptr;
        as->split = bufs.split[d];
        as->nsplit = as->splitctr;
        as->m = as->new_m;
        as->K = as->new_K;
        as->ntiles = (as->new_m + kTileEdges - 1) / kTileEdges;
        as->dst_arcs = d ^ 1u;
        as->do_copy = 0;
    }
    as->rowctr = 0;
    as->arcctr = 0;
    as->splitctr = 0;
    const bool small = handoff_arcs > 0 && as->m <= handoff_arcs && as->nnodes <= handoff_nodes;
    st->handoff = small ? 1u : 0u;
    st->active_nodes = as->nnodes;
    st->active_rows = as->K;
    st->active_arcs = (uint32_t)min(as->m, (uint64_t)0xffffffffu);
    if (use_handle) cudaGraphSetConditional(handle, small ? 0u : 1u);
}

// ---------------------------------------------------------------------------
// Node list and followers, built once per refinement after the initial pass.
// ---------------------------------------------------------------------------

// For every group of arc-less nodes with the same initial label: its smallest
// node (grep) and whether it has more than one member (gcnt, saturating at 2).
// Most such nodes share a handful of labels, so they are combined per warp
// (__match_any_sync), then per block in a small shared-memory table, and
// only then in global memory, where the words are read before any atomic:
// once a label's minimum and count are settled, later blocks only read.
constexpr int kRepSlots = 256;
constexpr int kRepProbes = 32;
static __global__ void __launch_bounds__(256) k_group_reps(uint32_t n, const uint64_t* __restrict__ off,
                                                           const uint32_t* __restrict__ initlab,
                                                           uint32_t* __restrict__ grep, uint32_t* __restrict__ gcnt)
{
    __shared__ uint32_t s_lab[kRepSlots], s_min[kRepSlots], s_cnt[kRepSlots];
    for (int i = threadIdx.x; i < kRepSlots; i += blockDim.x) {
        s_lab[i] = 0xffffffffu;
        s_min[i] = 0xffffffffu;
        s_cnt[i] = 0u;
    }
    __syncthreads();
    // grid-stride, 4 nodes per thread and step (their loads overlap): a block
    // combines all its stretches before touching the global words, so each
    // hot label sees one update per block, not per 256 nodes
    constexpr int U = 4;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x * U; base < n; base += stride * U) {
        bool dang[U];
        uint32_t lab[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + j * blockDim.x + threadIdx.x;
            dang[j] = u < n && off[u + 1] == off[u];
        }
#pragma unroll
        for (int j = 0; j < U; ++j) lab[j] = dang[j] ? initlab[base + j * blockDim.x + threadIdx.x] : 0u;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + j * blockDim.x + threadIdx.x;
            const unsigned dm = __ballot_sync(0xffffffffu, dang[j]);
            if (!dang[j]) continue;
            const uint32_t g = lab[j];
            const unsigned peers = __match_any_sync(dm, g);
            const uint32_t umin = __reduce_min_sync(peers, u);
            if ((threadIdx.x & 31) != (uint32_t)(__ffs(peers) - 1)) continue;
            // open-addressed shared table keyed by label; a key whose probe
            // sequence is full goes to the global words directly
            uint32_t h = (g * 0x9e3779b1u) >> 24;
            bool placed = false;
            for (int p = 0; p < kRepProbes && !placed; ++p, h = (h + 1) & (kRepSlots - 1)) {
                const uint32_t prev = atomicCAS(&s_lab[h], 0xffffffffu, g);
                if (prev == 0xffffffffu || prev == g) {
                    atomicMin(&s_min[h], umin);
                    atomicAdd(&s_cnt[h], (uint32_t)__popc(peers));
                    placed = true;
                }
            }
            if (!placed) {
                if (*(volatile uint32_t*)&grep[g] > umin) atomicMin(&grep[g], umin);
                if (*(volatile uint32_t*)&gcnt[g] < 2u) atomicAdd(&gcnt[g], (uint32_t)__popc(peers));
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRepSlots; i += blockDim.x) {
        const uint32_t g = s_lab[i];
        if (g == 0xffffffffu) continue;
        if (*(volatile uint32_t*)&grep[g] > s_min[i]) atomicMin(&grep[g], s_min[i]);
        if (*(volatile uint32_t*)&gcnt[g] < 2u) atomicAdd(&gcnt[g], s_cnt[i]);
    }
}

// Node list = non-singleton nodes that are not followers (representatives
// flagged); follower pairs; singleton count.  Grid-stride, both lists written
// through warp-private shared-memory buffers (warp_append: few reservations
// on the two counters, no block barrier per step).
static __global__ void __launch_bounds__(kNodeThreads) k_build_lists(uint32_t n, const uint64_t* __restrict__ off,
                                                                     const uint32_t* __restrict__ initlab,
                                                                     const uint32_t* __restrict__ col,
                                                                     const uint32_t* __restrict__ grep,
                                                                     const uint32_t* __restrict__ gcnt,
                                                                     ActiveSet* __restrict__ as, uint32_t* __restrict__ nodes,
                                                                     uint2* __restrict__ pairs)
{
    constexpr int W = kNodeThreads / 32;
    __shared__ uint32_t s_nodes[W][kWarpBuf];
    __shared__ uint2 s_pairs[W][kWarpBuf];
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    const uint32_t warp = threadIdx.x >> 5;
    uint32_t cn = 0, cp = 0;
    uint32_t singles = 0;
    // 4 nodes per thread and step: their dependent loads (offsets, then the
    // initial label, then the group words) overlap
    constexpr int U = 4;
    const uint32_t stride = gridDim.x * kNodeThreads;
    for (uint32_t base = blockIdx.x * kNodeThreads * U; base < n; base += stride * U) {
        bool single[U], dang[U];
        uint32_t g[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + j * kNodeThreads + threadIdx.x;
            single[j] = u < n && (col[u] & kSingleton) != 0;
            dang[j] = u < n && !single[j] && off[u + 1] == off[u];
        }
#pragma unroll
        for (int j = 0; j < U; ++j) g[j] = dang[j] ? initlab[base + j * kNodeThreads + threadIdx.x] : 0u;
        uint32_t gc[U], gr[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            gc[j] = dang[j] ? gcnt[g[j]] : 0u;
            gr[j] = dang[j] ? grep[g[j]] : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint32_t u = base + j * kNodeThreads + threadIdx.x;
            const bool valid = u < n;
            bool follower = false, rep = false;
            uint32_t r = 0;
            if (dang[j] && gc[j] >= 2u) {
                r = gr[j];
                follower = r != u;
                rep = r == u;
            }
            const bool listed = valid && !single[j] && !follower;
            singles += single[j] ? 1u : 0u;
            warp_append<uint32_t>(listed, u | (rep ? kRepFlag : 0u), s_nodes[warp], cn, &as->nodectr, nodes);
            warp_append<uint2>(follower, make_uint2(u, r), s_pairs[warp], cp, &as->nfollow, pairs);
        }
    }
    warp_append_flush<uint32_t>(s_nodes[warp], cn, &as->nodectr, nodes);
    warp_append_flush<uint2>(s_pairs[warp], cp, &as->nfollow, pairs);
    block_count<kNodeThreads>(singles, &as->retired, sm);
}

// Publishes the node list that k_build_lists wrote into buffer 0 (the next
// compaction writes buffer 1).
static __global__ void k_publish_list(ActiveSet* as)
{
    as->nnodes = as->nodectr;
    as->nodectr = 0;
    as->dst_nodes = 1;
}

// Zeroes the signatures of the given rows (the split rows of the whole-graph
// tiling, before a refinement starts on it: an earlier refinement may have
// left values there that the first pass would add to).
static __global__ void k_zero_rows(const uint32_t* __restrict__ list, uint32_t count, Sig* __restrict__ sig)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        sig_store(&sig[list[i]], 0ull, 0u);
    }
}

// Clears the table when the stamp wrapped.
__device__ __forceinline__ void clear_table_body(const RoundState* __restrict__ st, Entry* __restrict__ tab, uint64_t entries)
{
    if (!st->clear_pending) return;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += (uint64_t)gridDim.x * blockDim.x) {
        tab[i].k1 = 0ull;
        tab[i].hi = 0ull;
    }
}

__device__ __forceinline__ void clear_table_all(Entry* __restrict__ tab, uint64_t entries)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += (uint64_t)gridDim.x * blockDim.x) {
        tab[i].k1 = 0ull;
        tab[i].hi = 0ull;
    }
}

static __global__ void k_clear_table(const RoundState* __restrict__ st, Entry* __restrict__ tab, uint64_t entries)
{
    clear_table_body(st, tab, entries);
}

// ---------------------------------------------------------------------------
// Persistent pass kernel: once the active set is small, one cooperative
// launch runs the remaining passes (the same phases as the kernels above,
// separated by grid barriers) instead of a dozen small launches per pass.
// The barrier is a counter + generation word; every wait is bounded: after
// kBarrierSpin polls the kernel raises kErrBarrier and every block returns.
// ---------------------------------------------------------------------------
struct GridSync {
    unsigned count;
    unsigned gen;
};

constexpr uint32_t kBarrierSpin = 1u << 24;  // polls of ~64 ns: more than a second

__device__ __forceinline__ bool grid_barrier(GridSync* gs, RoundState* st)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &gs->gen;
        volatile uint32_t* verr = &st->error;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&gs->count, 1u) == gridDim.x - 1u) {
            gs->count = 0;  // nobody else touches the counter until the generation moves
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        } else {
            uint32_t it = 0;
            while (*vgen == g) {
                if (++it > kBarrierSpin || (*verr & kErrBarrier)) {
                    atomicOr(&st->error, kErrBarrier);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return !(*(volatile uint32_t*)&st->error & kErrBarrier);
}

struct PersistArgs {
    ActiveSet* as;
    RoundState* st;
    uint32_t* col;
    Sig* sig;
    Entry* tab;                  // the 16-byte stamped table (cleared when the stamp wraps)
    unsigned long long* tab8;    // the 8-byte list table (zeroed over the window every pass)
    int use8;                    // the passes use tab8: small windows, whose zeroing costs less than
                                 // the 16-byte table's extra load per insert
    uint32_t log2tab;
    uint64_t tab_entries;
    uint32_t* slot;
    const uint2* pairs;
    GridSync* gs;
    int weighted;
    uint32_t* joined;
};

// Signatures one row per lane, for active sets of short rows (the small tail,
// and a pass kernel's passes whose rows average at most 4 arcs): a warp takes
// 32 consecutive rows of the active arc set; each lane folds its row's arcs
// four at a time (rows of at most kRowLong arcs), and the rows longer than
// that are folded by the whole warp afterwards, one at a time (a strided loop
// and a shuffle reduction).  The sums are the tiled kernel's (wrap-around sums
// of the same per-arc terms, in another order), and every row is written
// whole, with no atomics.  Few registers: the persistent kernel that runs it
// keeps more warps resident than one built around the 16-arcs-per-lane tile
// fold.  NC false (the persistent kernel): colours are read at L2, since the
// same launch rewrites them between its phases; a pass kernel reads them
// through the read-only path.
constexpr uint32_t kRowLong = 32;
constexpr int kPersistBlocksPerSM = 4;  // 4 x 256 threads resident per SM (64 registers, no spills)

template <bool WEIGHTED, bool NC = false>
__device__ __forceinline__ void row_signature_body(const ActiveSet* __restrict__ as, const uint32_t* __restrict__ col,
                                                   Sig* __restrict__ sig, uint64_t salt)
{
    const uint32_t K = as->K;
    const bool r64 = as->roff64 != 0;
    const uint64_t* __restrict__ roff64 = reinterpret_cast<const uint64_t*>(as->roff);
    const uint32_t* __restrict__ roff32 = reinterpret_cast<const uint32_t*>(as->roff);
    const uint32_t* __restrict__ rows = as->rows;
    const uint32_t* __restrict__ idx = as->idx;
    const uint64_t* __restrict__ wt = as->wt;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t nwarps = gridDim.x * wpb;
    for (uint32_t base = (blockIdx.x * wpb + (threadIdx.x >> 5)) * 32u; base < K; base += nwarps * 32u) {
        const uint32_t k = base + lane;
        uint64_t b = 0, e = 0;
        uint32_t node = 0;
        if (k < K) {
            b = r64 ? roff64[k] : (uint64_t)roff32[k];
            e = r64 ? roff64[k + 1] : (uint64_t)roff32[k + 1];
            node = rows[k];  // issued beside the offsets: the store at the end waits for no load
        }
        const bool longrow = e - b > kRowLong;
        if (k < K && !longrow) {
            uint64_t s1 = 0;
            uint32_t s2 = 0;
            // four arcs at a time: their head loads, then their colour loads,
            // are issued side by side (one dependent pair per four arcs)
            for (uint64_t a = b; a < e; a += 4) {
                uint32_t h[4], c[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) h[j] = a + j < e ? idx[a + j] : 0u;
#pragma unroll
                for (int j = 0; j < 4; ++j) c[j] = a + j < e ? gather_col<NC>(col + h[j]) : 0u;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (a + j >= e) break;
                    uint64_t t1;
                    uint32_t t2;
                    arc_terms(c[j], salt, t1, t2);
                    if (WEIGHTED) {
                        const uint64_t w = wt[a + j];
                        t1 *= w;
                        t2 *= (uint32_t)w;
                    }
                    s1 += t1;
                    s2 += t2;
                }
            }
            sig_store(&sig[node], s1, s2);
        }
        unsigned lm = __ballot_sync(0xffffffffu, k < K && longrow);
        while (lm) {
            const int src = __ffs(lm) - 1;
            lm &= lm - 1u;
            const uint64_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
            uint64_t s1 = 0;
            uint32_t s2 = 0;
            for (uint64_t a = bb + lane; a < ee; a += 32) {
                uint64_t t1;
                uint32_t t2;
                arc_terms(gather_col<NC>(col + idx[a]), salt, t1, t2);
                if (WEIGHTED) {
                    const uint64_t w = wt[a];
                    t1 *= w;
                    t2 *= (uint32_t)w;
                }
                s1 += t1;
                s2 += t2;
            }
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                s1 += __shfl_xor_sync(0xffffffffu, s1, d);
                s2 += __shfl_xor_sync(0xffffffffu, s2, d);
            }
            if (lane == (uint32_t)src) sig_store(&sig[node], s1, s2);
        }
    }
}

// A pass's signatures by the shape of its active rows: one row per lane when
// they are short (at most 4 arcs on average, where a tile fold's lanes would
// each close several rows), else the 512-arc tile fold.  Both write the same
// sums.
template <bool WEIGHTED>
static __global__ void __launch_bounds__(kTileThreads) k_signature_auto(const ActiveSet* __restrict__ as,
                                                                        const RoundState* __restrict__ st,
                                                                        const uint32_t* __restrict__ col,
                                                                        Sig* __restrict__ sig)
{
    if (as->m <= 4ull * as->K) row_signature_body<WEIGHTED, true>(as, col, sig, pass_salt1(st->seed, st->round));
    else signature_body<WEIGHTED, uint32_t>(as, st, col, sig);
}

// Per pass: [table clear when the stamp wrapped] + signatures | inserts |
// relabel | [followers, only when a representative changed], three grid
// barriers (four with followers).  The clear may share the signature phase:
// the signatures do not touch the table, and the barrier after them orders
// the clear before every insert.  The end-of-pass decision (blocks counted,
// fixpoint, round limit) is taken by every block from its own copy of the pass
// state (round, stamp, previous count) and the counter of the pass, which is
// final after the insert barrier; counters and the representative flag come
// in pairs by pass parity, so block 0 can reset the next pass's pair while
// other blocks still read this pass's.  Block 0 mirrors the state into
// RoundState for the host.
// ROWS: the signature phase folds one row per lane (short rows; fewer
// registers, kPersistBlocksPerSM blocks per SM); otherwise it runs the
// 512-arc tile fold of k_signature (load-balanced for long rows; 3 blocks per
// SM).  Both write the same sums.
template <bool ROWS>
static __global__ void __launch_bounds__(kNodeThreads, ROWS ? kPersistBlocksPerSM : 3) k_refine_persistent(PersistArgs a)
{
    static_assert(kNodeThreads == kTileThreads, "the tile fold runs one tile per warp");
    __shared__ BlockReserveSmem<kNodeThreads> sm;
    RoundState* st = a.st;
    uint32_t round = st->round, stamp = st->stamp, prev = st->prev;
    bool clear = st->clear_pending != 0u;
    const uint32_t max_rounds = st->max_rounds;
    const uint32_t retired = a.as->retired;
    const uint64_t seed = st->seed;
    for (;;) {
        const uint32_t p = round & 1u;
        if (clear) clear_table_all(a.tab, a.tab_entries);
        if (a.use8) clear_window8(a.as, a.tab8, a.log2tab);
        if (ROWS) {
            if (a.weighted) row_signature_body<true>(a.as, a.col, a.sig, pass_salt1(seed, round));
            else row_signature_body<false>(a.as, a.col, a.sig, pass_salt1(seed, round));
        } else {
            const TileRange all{0u, 0u, nullptr, nullptr, 0ull};
            if (a.weighted) signature_body<true, uint32_t, false>(a.as, st, a.col, a.sig, all, nullptr, nullptr, round);
            else signature_body<false, uint32_t, false>(a.as, st, a.col, a.sig, all, nullptr, nullptr, round);
        }
        if (!grid_barrier(a.gs, st)) return;
        const uint32_t made =
            a.use8 ? insert_list_body<unsigned long long>(a.as, st, a.col, a.sig, a.tab8, a.log2tab, a.slot, a.joined, round, stamp, prev)
                   : insert_list_body<Entry>(a.as, st, a.col, a.sig, a.tab, a.log2tab, a.slot, a.joined, round, stamp, prev);
        block_count<kNodeThreads>(made, &st->pcount[p], sm);
        if (!grid_barrier(a.gs, st)) return;
        if (a.use8) relabel_list_body<false, unsigned long long>(a.as, st, a.col, a.tab8, a.slot, a.sig, a.joined, round, &st->prep[p]);
        else relabel_list_body<false, Entry>(a.as, st, a.col, a.tab, a.slot, a.sig, a.joined, round, &st->prep[p]);
        if (!grid_barrier(a.gs, st)) return;
        if (*(volatile uint32_t*)&st->prep[p]) {
            follow_body(a.as, st, a.pairs, a.col, &st->prep[p]);
            if (!grid_barrier(a.gs, st)) return;
        }
        const uint32_t cnt = *(volatile uint32_t*)&st->pcount[p] + retired;
        const bool done = cnt == prev;
        ++round;
        prev = cnt;
        stamp = stamp % 255u + 1u;
        clear = stamp == 1u;
        const bool over = !done && round >= max_rounds;
        const bool err = *(volatile uint32_t*)&st->error != 0u;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->round = round;
            if (round < kRoundLog) st->round_blocks[round] = cnt;
            st->prev = cnt;
            st->stamp = stamp;
            st->clear_pending = clear ? 1u : 0u;
            st->count = 0u;
            st->rep_changed = 0u;
            st->pcount[p ^ 1u] = 0u;
            st->prep[p ^ 1u] = 0u;
            if (done) st->done = 1u;
            if (over) atomicOr(&st->error, kErrRounds);
        }
        if (done || over || err) return;
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
