// lump64.cu -- exact lumping with double weights.
//
// Valmari's minimiser built with MDP_weight_is_double (src/part_ref/MDPmin.cc:37,
// 107-113; its splitter loop MDP_minimize.cc:567-637) lumps a chain whose
// transition weights are doubles: the weight of a state into a block is the
// double sum of its transitions into the block, rounded to float
// (MDP_round_weight) before any comparison, and a sum that rounds to zero
// counts as no transition (MDP_minimize.cc:596-599).  The coarsest partition
// that refines the initial one and in which the members of every block have
// equal rounded sums into every block is what this module computes.
//
// Signature passes, as the integer path, but the signature of a node is no
// longer a sum of per-arc terms (a float-rounded sum is not additive), so a
// pass first groups the arcs by (successor block, row):
//   1. k_l64_rep_flags + a scan + k_l64_block_ids: the dense id of every
//      block (its rank among the blocks' smallest nodes), per node;
//   2. k_l64_keys: one 64-bit key per arc, (block id of its head << lb) | row,
//      carrying the arc's weight;
//   3. the stable radix sort (radix.cuh) on the block-id bits only (the
//      rows are in order already and the sort is stable): arcs grouped by
//      (block, row), in arc order inside a group.  The first pass of a
//      uniform start (one block) sorts nothing;
//   4. k_l64_sums: the thread of a group's first position adds its weights in
//      arc order (double, read in sorted order; a warp per group of more than
//      32 arcs, k_l64_long_sums), rounds the sum to float; a nonzero sum adds
//      the hash of (block, float bits) to the row's signature (wrap-around 64
//      + 32-bit sums, so the order of the adds does not matter; neighbouring
//      groups belong to different rows);
//   5. k_l64_insert + k_l64_relabel: classes of (label, signature) in the
//      stamped 16-byte relabel table of the integer path, new label = smallest
//      member;
//   6. the host reads the class count: unchanged = fixpoint.
// Exact check at the fixpoint (the groups of the last pass are those of the
// final partition, whose canonical labels the pass left unchanged): the
// nonzero groups are compacted and re-sorted by row (stable, row bits only),
// and every node's list of (block, float bits) must equal that of its
// block's smallest node.  Nodes that differ are split off (key =
// (label, failed)) and the passes resume; the result is returned only once
// the check passed.  Weights must be finite with magnitude below 2^960 (so no
// sum of up to 2^32 of them overflows a double).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "common.cuh"
#include "internal.h"
#include "radix.cuh"
#include "scan.cuh"

using namespace rbsc;

namespace {

constexpr int kT = 256;

unsigned grid_of(uint64_t n, unsigned t = kT)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + t - 1) / t, 148ull * 64));
}

// Device counters of one call.
struct L64Counters {
    uint32_t classes;  // classes made by the last insert
    uint32_t failed;   // nodes that failed the exact check
    uint32_t nonzero;  // groups with a nonzero rounded sum
    uint32_t error;    // kErr* bits
    uint32_t long_groups;  // groups of more than kShortGroup arcs, listed for k_l64_long_sums
    uint32_t pad[3];
};

constexpr uint32_t kL64BadWeight = 32u;  // a weight that is not finite or not below 2^960

// 0 for a finite weight below 2^960 in magnitude
__global__ void k_l64_check_weights(uint64_t m, const double* __restrict__ w, L64Counters* __restrict__ c)
{
    bool bad = false;
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x)
        bad |= !(fabs(w[a]) < 0x1p960);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&c->error, kL64BadWeight);
}

// row of every arc: one warp per row
__global__ void k_l64_rows(uint32_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ src)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t u = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); u < n; u += warps)
        for (uint64_t a = off[u] + lane; a < off[u + 1]; a += 32) src[a] = (uint32_t)u;
}

// flag[u] = u is the smallest node of its block
__global__ void k_l64_rep_flags(uint32_t n, const uint32_t* __restrict__ col, uint32_t* __restrict__ flag)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        flag[u] = col[u] == (uint32_t)u ? 1u : 0u;
}

// bid[u] = dense id of u's block (rank[] = exclusive scan of the flags)
__global__ void k_l64_block_ids(uint32_t n, const uint32_t* __restrict__ col, const uint32_t* __restrict__ rank,
                                uint32_t* __restrict__ bid)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x)
        bid[u] = rank[col[u]];
}

__global__ void k_l64_keys(uint64_t m, uint32_t lb, const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx,
                           const uint32_t* __restrict__ bid, const unsigned long long* __restrict__ w,
                           unsigned long long* __restrict__ keys, unsigned long long* __restrict__ vals)
{
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x) {
        keys[a] = ((unsigned long long)bid[idx[a]] << lb) | src[a];
        vals[a] = w[a];
    }
}

__device__ __forceinline__ void group_hash(uint32_t lab, uint32_t bits, uint64_t salt1, uint32_t salt2, uint64_t& h1,
                                           uint32_t& h2)
{
    h1 = fmix64((((uint64_t)lab << 32) | bits) ^ salt1);
    h2 = fmix32((lab * 0x9e3779b1u) ^ fmix32(bits ^ salt2));
}

// The rounded sum of one group, its bits and its signature term.
__device__ __forceinline__ void group_done(uint64_t g, double s, unsigned long long k, uint32_t lb, uint64_t salt1,
                                           uint32_t salt2, int hash_bits, Sig* __restrict__ sig, uint32_t* __restrict__ bits)
{
    const float f = __double2float_rn(s);
    const uint32_t fb = f != 0.0f ? __float_as_uint(f) : 0u;
    bits[g] = fb;
    if (fb) {
        uint64_t h1;
        uint32_t h2;
        group_hash((uint32_t)(k >> lb), fb, salt1, salt2, h1, h2);
        if (hash_bits) {  // test hook: truncated (or no) signatures
            h1 = (hash_bits >= 64 || hash_bits < 0) ? 0ull : (h1 & ((1ull << hash_bits) - 1ull));
            h2 = 0u;
        }
        const uint32_t row = (uint32_t)(k & ((1ull << lb) - 1ull));
        atomicAdd(&sig[row].s1, (unsigned long long)h1);
        atomicAdd(&sig[row].s2, h2);
    }
}

// One thread per sorted position; the first position of each (block, row)
// group adds the group's weights in arc order (the sort kept it) in double and
// rounds the sum to float.  bits[i] = the float's bits at a group's first
// position (0 for a sum that rounds to zero, of either sign: the group adds
// nothing), 0 at every other position.  Groups of more than kShortGroup arcs
// are listed (by first position) for k_l64_long_sums.
constexpr uint32_t kShortGroup = 32;

__global__ void k_l64_sums(L64Counters* __restrict__ c, uint64_t m, uint32_t lb, const unsigned long long* __restrict__ keys,
                           const unsigned long long* __restrict__ vals, uint64_t salt1, uint32_t salt2, int hash_bits,
                           Sig* __restrict__ sig, uint32_t* __restrict__ bits, uint32_t* __restrict__ long_list)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (i > 0 && keys[i - 1] == k) {
            bits[i] = 0u;
            continue;
        }
        const uint64_t end = min(m, i + kShortGroup + 1);
        double s = 0.0;
        uint64_t j = i;
        for (; j < end && keys[j] == k; ++j) s += __longlong_as_double((long long)vals[j]);
        if (j - i > kShortGroup) {
            long_list[atomicAdd(&c->long_groups, 1u)] = (uint32_t)i;
            continue;
        }
        group_done(i, s, k, lb, salt1, salt2, hash_bits, sig, bits);
    }
}

// One warp per long group: the lanes load 32 keys and weights at a time (the
// next 32 while lane 0 adds the current ones, handed over by shuffles in lane
// order), so the sum is the same arc-order double sum as k_l64_sums', at the
// pace of the dependent adds rather than of one load per weight.
__global__ void __launch_bounds__(kT) k_l64_long_sums(const L64Counters* __restrict__ c, uint64_t m, uint32_t lb,
                                                      const unsigned long long* __restrict__ keys,
                                                      const unsigned long long* __restrict__ vals, uint64_t salt1,
                                                      uint32_t salt2, int hash_bits, Sig* __restrict__ sig,
                                                      uint32_t* __restrict__ bits, const uint32_t* __restrict__ long_list)
{
    const uint32_t L = c->long_groups;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t t = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); t < L; t += warps) {
        const uint64_t b = long_list[t];
        const unsigned long long k = keys[b];
        double s = 0.0;
        bool in = b + lane < m && keys[b + lane] == k;
        double x = in ? __longlong_as_double((long long)vals[b + lane]) : 0.0;
        for (uint64_t a0 = b;; a0 += 32) {
            // the group is contiguous: its lanes of this chunk are a prefix
            const uint32_t cnt = (uint32_t)__popc(__ballot_sync(0xffffffffu, in));
            const uint64_t a1 = a0 + 32;
            const bool nin = cnt == 32u && a1 + lane < m && keys[a1 + lane] == k;
            const double nx = nin ? __longlong_as_double((long long)vals[a1 + lane]) : 0.0;
            for (uint32_t j = 0; j < cnt; ++j) {
                const double v = __shfl_sync(0xffffffffu, x, j);
                if (lane == 0) s += v;
            }
            if (cnt < 32u) break;
            in = nin;
            x = nx;
        }
        if (lane == 0) group_done(b, s, k, lb, salt1, salt2, hash_bits, sig, bits);
    }
}

// Class of every node by key: MODE 0 = (label, signature) hashed, 1 = the
// initial colour (init may be null: one class), 2 = (label, failed flag).
template <int MODE>
__global__ void k_l64_insert(uint32_t n, const uint32_t* __restrict__ col, const Sig* __restrict__ sig,
                             const uint32_t* __restrict__ aux, uint64_t seed, uint32_t stamp, Entry* __restrict__ tab,
                             uint32_t log2size, uint32_t* __restrict__ slot, L64Counters* __restrict__ c)
{
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += (uint64_t)gridDim.x * blockDim.x) {
        const bool need = base + (threadIdx.x & 31) < n;
        const uint32_t u = (uint32_t)(base + (threadIdx.x & 31));
        uint64_t k1 = 0;
        uint32_t k2 = stamp;
        if (need) {
            if (MODE == 0) {
                const uint32_t lab = col[u];
                k1 = sig[u].s1 ^ fmix64(((uint64_t)lab << 1 | 1ull) * kGolden ^ seed);
                k2 = ((sig[u].s2 ^ fmix32(lab * 0x9e3779b1u + (uint32_t)seed)) & 0xffffff00u) | stamp;
            } else if (MODE == 1) {
                k1 = aux ? (uint64_t)aux[u] : 0ull;
            } else {
                k1 = (uint64_t)col[u] | ((uint64_t)(aux[u] != 0u) << 32);
            }
        }
        bool nb = false;
        insert_warp(need, u, u, false, k1, k2, stamp, tab, log2size, slot, &c->error, nb);
        count_blocks(nb, &c->classes);
    }
}

__global__ void k_l64_relabel(uint32_t n, const Entry* __restrict__ tab, const uint32_t* __restrict__ slot,
                              uint32_t* __restrict__ col)
{
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t* v = reinterpret_cast<const uint32_t*>(tab + slot[u]) + 3;
        col[u] = __ldg(v) & kLabelMask;
    }
}

// nzflag[i] = position i starts a group with a nonzero rounded sum
__global__ void k_l64_nz_flags(uint64_t m, const uint32_t* __restrict__ bits, uint32_t* __restrict__ nzflag)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        nzflag[i] = bits[i] != 0u ? 1u : 0u;
}

// the nonzero groups, compacted: ckey = (row << cw) | block id, cval = float
// bits; cnt[row] counts them (zeroed before)
__global__ void k_l64_nz_compact(uint64_t m, uint32_t lb, uint32_t cw, const unsigned long long* __restrict__ keys,
                                 const uint32_t* __restrict__ bits, const uint32_t* __restrict__ nzpos,
                                 unsigned long long* __restrict__ ckey, uint32_t* __restrict__ cval, uint32_t* __restrict__ cnt)
{
    const uint64_t mask = (1ull << lb) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        if (bits[i]) {
            const unsigned long long k = keys[i];
            const uint32_t row = (uint32_t)(k & mask);
            const uint32_t p = nzpos[i];
            ckey[p] = ((unsigned long long)row << cw) | (k >> lb);
            cval[p] = bits[i];
            atomicAdd(&cnt[row], 1u);
        }
}

// fail[u] = u's (block, float bits) list differs from its block's smallest
// node's; the lists are the row-sorted compacted groups [first[u], first[u+1])
__global__ void k_l64_check(uint32_t n, uint32_t cw, const uint32_t* __restrict__ col, const uint32_t* __restrict__ first,
                            const unsigned long long* __restrict__ ckey, const uint32_t* __restrict__ cval,
                            uint32_t* __restrict__ fail, L64Counters* __restrict__ c)
{
    const unsigned long long bmask = (1ull << cw) - 1ull;
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = col[u];
        bool bad = false;
        if (r != u) {
            const uint32_t bu = first[u], eu = first[u + 1], br = first[r], er = first[r + 1];
            bad = eu - bu != er - br;
            for (uint32_t i = 0; !bad && i < eu - bu; ++i)
                bad = (ckey[bu + i] & bmask) != (ckey[br + i] & bmask) || cval[bu + i] != cval[br + i];
        }
        fail[u] = bad ? 1u : 0u;
        if (bad) atomicAdd(&c->failed, 1u);
    }
}

}  // namespace

extern "C" rbsc_status rbsc_refine_f64(rbsc_ctx* ctx, const rbsc_csr* host_graph, const double* weights,
                                       const uint32_t* init_colors, uint32_t* out_labels, rbsc_stats* stats)
{
    if (!ctx || !host_graph) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    if (host_graph->weights)
        return rbsc_fail(ctx, RBSC_ERR_INVALID, "rbsc_refine_f64: the weights are the double array, not host_graph->weights");
    if (host_graph->m && !weights) return rbsc_fail(ctx, RBSC_ERR_INVALID, "rbsc_refine_f64: null weights");
    if (host_graph->n && !out_labels) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null output");
    if (host_graph->m > 0xffffffffull) return rbsc_fail(ctx, RBSC_ERR_INVALID, "rbsc_refine_f64: more than 2^32 - 1 arcs");
    if (host_graph->n > (1u << 31)) return rbsc_fail(ctx, RBSC_ERR_INVALID, "rbsc_refine_f64: more than 2^31 nodes");
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof *stats);
    const uint64_t lc0 = rbsc::launch_counter();
    // the doubles travel as the 8-byte weights of the upload (which checks
    // offsets and heads); k_l64_check_weights checks their values
    rbsc_csr c = *host_graph;
    c.weights = reinterpret_cast<const uint64_t*>(weights);
    rbsc_graph* g = nullptr;
    EKS(rbsc_graph_upload(ctx, &c, &g));
    struct FreeG { rbsc_graph*& g; ~FreeG() { rbsc_graph_free(g); } } guard_g{g};
    cudaStream_t s = ctx->stream;
    const uint32_t N = g->n;
    const uint64_t M = g->m;
    if (N == 0) {
        if (stats) {
            stats->done = 1;
            stats->verified = 1;
        }
        return RBSC_OK;
    }
    const double* w = reinterpret_cast<const double*>(g->d_wt);
    Scratch sc(ctx);
    const auto bits_of = [](uint64_t v) -> uint32_t { return v ? 64u - (uint32_t)__builtin_clzll(v) : 0u; };
    const uint32_t lb = std::max(1u, bits_of(N - 1u));  // row bits of a key
    uint32_t log2tab = 10;
    while (log2tab < 33 && (1ull << log2tab) < 2ull * N) ++log2tab;
    uint32_t *col = nullptr, *slot = nullptr, *fail = nullptr, *first = nullptr, *bid = nullptr, *src = nullptr,
             *gid = nullptr, *bits = nullptr, *cval = nullptr, *cval_alt = nullptr;
    unsigned long long *keys = nullptr, *keys_alt = nullptr, *vals = nullptr, *vals_alt = nullptr;
    Sig* sig = nullptr;
    Entry* tab = nullptr;
    L64Counters* dc = nullptr;
    void* tmp = nullptr;
    EKS(sc.get(&col, N));
    EKS(sc.get(&slot, N));
    EKS(sc.get(&fail, N));
    EKS(sc.get(&first, (size_t)N + 1));
    EKS(sc.get(&bid, N));
    EKS(sc.get(&sig, N));
    EKS(sc.get(&tab, (size_t)1 << log2tab));
    EKS(sc.get(&dc, 1));
    EKS(sc.get(&src, M));
    EKS(sc.get(&keys, M));
    EKS(sc.get(&keys_alt, M));
    EKS(sc.get(&vals, M));
    EKS(sc.get(&vals_alt, M));
    EKS(sc.get(&gid, M + 1));
    EKS(sc.get(&bits, M));
    EKS(sc.get(&cval, M));
    EKS(sc.get(&cval_alt, M));
    const uint64_t big = std::max<uint64_t>(M, N) + 1;
    EKS(sc.get((char**)&tmp, std::max(radix_temp_bytes(M), scan_temp_bytes<uint32_t>(big)) + 1024));
    EK(cudaMemsetAsync(dc, 0, sizeof(L64Counters), s));
    EK(cudaMemsetAsync(tab, 0, sizeof(Entry) << log2tab, s));
    ++rbsc::launch_counter();
    k_l64_check_weights<<<grid_of(M), kT, 0, s>>>(M, w, dc);
    ++rbsc::launch_counter();
    k_l64_rows<<<grid_of(32ull * N), kT, 0, s>>>(N, g->d_off, src);
    EK(cudaGetLastError());

    // the initial colours' classes in the table (stamp 1), canonical labels
    uint32_t* d_init = nullptr;
    if (init_colors) {
        EKS(sc.get(&d_init, N));
        EK(cudaMemcpyAsync(d_init, init_colors, 4ull * N, cudaMemcpyHostToDevice, s));
    }
    uint32_t stamp = 1;
    L64Counters hc{};
    auto read_counters = [&]() -> rbsc_status {
        EK(cudaMemcpyAsync(&hc, dc, sizeof hc, cudaMemcpyDeviceToHost, s));
        EK(cudaStreamSynchronize(s));
        if (hc.error & kL64BadWeight)
            return rbsc_fail(ctx, RBSC_ERR_INVALID, "rbsc_refine_f64: a weight is not finite or not below 2^960 in magnitude");
        if (hc.error & kErrProbe) return rbsc_fail(ctx, RBSC_ERR_DEVICE, "relabel table overflow");
        return RBSC_OK;
    };
    // classes of one insert (the counter zeroed first), then the new labels
    auto relabel = [&](int mode, const uint32_t* aux) -> rbsc_status {
        EK(cudaMemsetAsync(&dc->classes, 0, 4, s));
        ++rbsc::launch_counter();
        if (mode == 0)
            k_l64_insert<0><<<grid_of(N), kT, 0, s>>>(N, col, sig, aux, ctx->opts.seed, stamp, tab, log2tab, slot, dc);
        else if (mode == 1)
            k_l64_insert<1><<<grid_of(N), kT, 0, s>>>(N, col, sig, aux, ctx->opts.seed, stamp, tab, log2tab, slot, dc);
        else
            k_l64_insert<2><<<grid_of(N), kT, 0, s>>>(N, col, sig, aux, ctx->opts.seed, stamp, tab, log2tab, slot, dc);
        ++rbsc::launch_counter();
        k_l64_relabel<<<grid_of(N), kT, 0, s>>>(N, tab, slot, col);
        EK(cudaGetLastError());
        // next stamp; the table is cleared when it wraps
        stamp = stamp % 255u + 1u;
        if (stamp == 1u) EK(cudaMemsetAsync(tab, 0, sizeof(Entry) << log2tab, s));
        return RBSC_OK;
    };
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1];
    EK(cudaEventRecord(e0, s));
    EKS(relabel(1, d_init));
    EKS(read_counters());
    uint32_t prev = hc.classes;
    const uint32_t initial_blocks = prev;
    std::vector<uint32_t> round_blocks{prev};
    const uint32_t max_rounds = ctx->opts.max_rounds ? ctx->opts.max_rounds : N + 1u;
    uint32_t rounds = 0, repairs = 0;
    bool verified = false;
    const int hash_bits = ctx->opts.test_hash_bits;
    const unsigned long long* w64 = reinterpret_cast<const unsigned long long*>(g->d_wt);
    const unsigned long_grid = (unsigned)ctx->sm_count * 8;
    for (;;) {
        // one signature pass; prev = the current number of blocks
        const uint32_t cb = bits_of(prev - 1u);  // block-id bits of a key
        bool in_alt = false;
        if (M) {
            ++rbsc::launch_counter();
            k_l64_rep_flags<<<grid_of(N), kT, 0, s>>>(N, col, first);
            EK((exclusive_scan<uint32_t, uint32_t>(first, first, N, (uint32_t*)nullptr, tmp, s)));
            ++rbsc::launch_counter();
            k_l64_block_ids<<<grid_of(N), kT, 0, s>>>(N, col, first, bid);
            ++rbsc::launch_counter();
            k_l64_keys<<<grid_of(M), kT, 0, s>>>(M, lb, src, g->d_idx, bid, w64, keys, vals);
            EK(cudaGetLastError());
            EK(radix_sort<unsigned long long>(keys, keys_alt, vals, vals_alt, M, (int)lb, (int)(lb + cb), tmp, s, &in_alt));
        }
        const unsigned long long* sk = in_alt ? keys_alt : keys;
        const unsigned long long* sv = in_alt ? vals_alt : vals;
        EK(cudaMemsetAsync(sig, 0, sizeof(Sig) * N, s));
        EK(cudaMemsetAsync(&dc->long_groups, 0, 4, s));
        if (M) {
            const uint64_t salt1 = pass_salt1(ctx->opts.seed, rounds);
            const uint32_t salt2 = pass_salt2(ctx->opts.seed, rounds);
            ++rbsc::launch_counter();
            k_l64_sums<<<grid_of(M), kT, 0, s>>>(dc, M, lb, sk, sv, salt1, salt2, hash_bits, sig, bits, cval_alt);
            ++rbsc::launch_counter();
            k_l64_long_sums<<<long_grid, kT, 0, s>>>(dc, M, lb, sk, sv, salt1, salt2, hash_bits, sig, bits, cval_alt);
            EK(cudaGetLastError());
        }
        EKS(relabel(0, nullptr));
        EKS(read_counters());
        ++rounds;
        round_blocks.push_back(hc.classes);
        if (hc.classes != prev) {
            prev = hc.classes;
            if (rounds >= max_rounds)
                return rbsc_fail(ctx, RBSC_ERR_NOT_CONVERGED, "no fixpoint after %u passes", rounds);
            continue;
        }
        if (!ctx->opts.verify) break;
        // exact check over this pass's groups (the final partition's): the
        // nonzero ones compacted into the key buffers the sort did not end in,
        // then sorted by row (stable: block order kept inside a row)
        unsigned long long* ck = in_alt ? keys : keys_alt;
        unsigned long long* ck_alt = in_alt ? keys_alt : keys;
        const uint32_t cw = std::max(1u, cb);
        EK(cudaMemsetAsync(first, 0, 4ull * (N + 1), s));
        EK(cudaMemsetAsync(&dc->failed, 0, 4, s));
        EK(cudaMemsetAsync(&dc->nonzero, 0, 4, s));
        const uint32_t* cv = cval;
        if (M) {
            ++rbsc::launch_counter();
            k_l64_nz_flags<<<grid_of(M), kT, 0, s>>>(M, bits, gid);
            EK((exclusive_scan<uint32_t, uint32_t>(gid, gid, M, (uint32_t*)nullptr, tmp, s)));
            ++rbsc::launch_counter();
            k_l64_nz_compact<<<grid_of(M), kT, 0, s>>>(M, lb, cw, sk, bits, gid, ck, cval, first);
            EK(cudaGetLastError());
            // nonzero groups = the per-row counts' total (read back for the sort's size)
            EK((exclusive_scan<uint32_t, uint32_t>(first, first, (uint64_t)N + 1, &dc->nonzero, tmp, s)));
            EKS(read_counters());
            bool c_alt = false;
            EK(radix_sort<uint32_t>(ck, ck_alt, cval, cval_alt, hc.nonzero, (int)cw, (int)(cw + lb), tmp, s, &c_alt));
            if (c_alt) {
                ck = ck_alt;
                cv = cval_alt;
            }
        } else {
            EK((exclusive_scan<uint32_t, uint32_t>(first, first, (uint64_t)N + 1, (uint32_t*)nullptr, tmp, s)));
        }
        ++rbsc::launch_counter();
        k_l64_check<<<grid_of(N), kT, 0, s>>>(N, cw, col, first, ck, cv, fail, dc);
        EK(cudaGetLastError());
        EKS(read_counters());
        if (hc.failed == 0) {
            verified = true;
            break;
        }
        // split the failed nodes off their blocks and refine on
        ++repairs;
        EKS(relabel(2, fail));
        EKS(read_counters());
        prev = hc.classes;
        if (rounds >= max_rounds) return rbsc_fail(ctx, RBSC_ERR_NOT_CONVERGED, "no fixpoint after %u passes", rounds);
    }
    EK(cudaEventRecord(e1, s));
    EK(cudaMemcpyAsync(out_labels, col, 4ull * N, cudaMemcpyDeviceToHost, s));
    EK(cudaStreamSynchronize(s));
    float dev_ms = 0.f;
    cudaEventElapsedTime(&dev_ms, e0, e1);
    if (stats) {
        stats->rounds = rounds;
        stats->blocks = prev;
        stats->done = 1;
        stats->verified = verified ? 1u : 0u;
        stats->repairs = repairs;
        stats->initial_blocks = initial_blocks;
        stats->device_ms = dev_ms;
        for (size_t i = 0; i < round_blocks.size() && i < 64; ++i) stats->round_blocks[i] = round_blocks[i];
        stats->kernel_launches = rbsc::launch_counter() - lc0;
        stats->h2d_bytes = 8ull * (N + 1) + 12ull * M + (init_colors ? 4ull * N : 0ull);
        stats->d2h_bytes = 4ull * N;
        stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return RBSC_OK;
}
