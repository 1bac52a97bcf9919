// noalloc.cu -- refinement of a small graph without any device allocation.
//
// Some callers cannot call cudaMalloc at all: code that runs while another
// framework owns the device memory pool, real-time paths that must not take
// the implicit device synchronisation an allocation can cause, or hosts that
// hand this library only pointers into memory they manage themselves.  For
// them rbsc_refine_noalloc refines a small graph (N <= 16384 nodes) in ONE
// kernel launch on the caller's stream.  Inputs and outputs are the caller's
// device buffers; every other byte the kernel needs lives in one file-scope
// __device__ array (g_noalloc_scratch, about 5 MB), which every GPU that loads
// this library holds until the process exits.
//
// The kernel is one thread block.  It computes the same partition as the
// multi-kernel path (hashed rounds to the fixpoint, then an exact check that
// splits any wrongly merged class and resumes), so its labels and counts equal
// those of rbsc_refine on the same graph.  The exact check here compares each
// node's row with its block representative's by counting colours in a
// per-warp array instead of sorting.
//
// Sharing rules: all calls share the scratch array.  The kernel clears what it
// needs at the start of every call; two calls whose kernels overlap on the GPU
// (different streams, no ordering between them) race on it and give wrong
// results.  The first call on a device resolves the array's device address with
// cudaGetSymbolAddress (with that device current) and keeps it until the
// process exits; make that first call before any stream capture that would
// include it, and make no call on a device after cudaDeviceReset on it.
//
// Unlike the reference (which trusts its input, rbsc.cu:156-180), the kernel
// checks the graph before its first indexed read, as the regular path's
// k_validate does: a malformed graph returns RBSC_ERR_INVALID in d_result.
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "common.cuh"
#include "refine_kernels.cuh"

using namespace rbsc;

namespace {

constexpr uint32_t kNaMaxNodes = RBSC_NOALLOC_MAX_NODES;
constexpr uint32_t kNaThreads = 1024;
constexpr uint32_t kNaWarps = kNaThreads / 32;
constexpr uint32_t kNaLog2Table = 15;  // 2^15 entries >= 2 * kNaMaxNodes

// scratch layout (byte offsets, all 256-aligned)
constexpr size_t kNaCol = 0;
constexpr size_t kNaInit = kNaCol + 4ull * kNaMaxNodes;
constexpr size_t kNaSig1 = kNaInit + 4ull * kNaMaxNodes;
constexpr size_t kNaSig2 = kNaSig1 + 8ull * kNaMaxNodes;
constexpr size_t kNaSlot = kNaSig2 + 4ull * kNaMaxNodes;
constexpr size_t kNaFail = kNaSlot + 4ull * kNaMaxNodes;
constexpr size_t kNaTable = kNaFail + 4ull * kNaMaxNodes;
constexpr size_t kNaCount = kNaTable + sizeof(Entry) * (1ull << kNaLog2Table);
constexpr size_t kNaBytes = kNaCount + 8ull * kNaWarps * kNaMaxNodes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

__device__ __forceinline__ uint64_t na_off(const void* off, int off64, uint32_t u)
{
    return off64 ? reinterpret_cast<const uint64_t*>(off)[u] : (uint64_t)reinterpret_cast<const uint32_t*>(off)[u];
}

// One table pass over all nodes with exact or hashed keys; returns the block
// count (new classes + singletons) to every thread.  mode 0 = hashed
// (signature), 1 = initial colour, 2 = repair (label, failure flag).
__device__ uint32_t na_table_pass(int mode, uint32_t n, uint32_t* col, const uint32_t* init, const unsigned long long* sig1,
                                  const uint32_t* sig2, const uint32_t* fail, Entry* tab, uint32_t log2tab, uint32_t* slot,
                                  uint64_t seed, uint32_t hash_bits, uint32_t* s_count, uint32_t* s_err)
{
    const uint32_t T = 1u << log2tab;
    for (uint32_t i = threadIdx.x; i < T; i += kNaThreads) {
        tab[i].k1 = 0ull;
        tab[i].hi = 0ull;
    }
    if (threadIdx.x == 0) *s_count = 0;
    __syncthreads();
    const uint32_t stamp = 1;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = warp * 32; base < n; base += kNaThreads) {
        const uint32_t u = base + lane;
        const bool active = u < n;
        const uint32_t c = active ? (mode == 1 ? 0u : col[u]) : kSingleton;
        const bool need = active && !(c & kSingleton);
        uint64_t k1 = 0;
        uint32_t k2 = stamp;
        if (need) {
            const uint32_t lab = c & kLabelMask;
            if (mode == 0) {
                uint64_t s1 = sig1[u];
                uint32_t s2 = sig2[u];
                if (hash_bits) {  // test hook: truncated (or, from 64 bits on, no) signatures
                    s1 = (hash_bits >= 64) ? 0ull : (s1 & ((1ull << hash_bits) - 1ull));
                    s2 = 0;
                }
                k1 = s1 ^ fmix64(((uint64_t)lab << 1 | 1ull) * kGolden ^ seed);
                k2 = ((s2 ^ fmix32(lab * 0x9e3779b1u + (uint32_t)seed)) & 0xffffff00u) | stamp;
            } else if (mode == 1) {
                k1 = init[u];
            } else {
                k1 = (uint64_t)lab | ((uint64_t)(fail[u] != 0u) << 32);
            }
        }
        bool nb = active && !need;
        insert_warp(need, u, u, false, k1, k2, stamp, tab, log2tab, slot, s_err, nb);
        const unsigned m = __ballot_sync(0xffffffffu, nb);
        if (lane == 0 && m) atomicAdd(s_count, (uint32_t)__popc(m));
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) {
        const uint32_t c = mode == 1 ? 0u : col[u];
        if (!(c & kSingleton)) col[u] = relabel_one<false>(c, tab, slot[u]);
    }
    __syncthreads();
    return *(volatile uint32_t*)s_count;
}

struct NaArgs {
    uint32_t n;
    uint64_t m;
    const void* off;
    int off64;
    const uint32_t* idx;
    const uint64_t* wt;
    const uint32_t* init;
    uint32_t* out;
    rbsc_noalloc_result* result;
    unsigned char* scratch;
    uint64_t seed;
    uint32_t max_rounds;
    uint32_t hash_bits;
};

static __global__ void __launch_bounds__(kNaThreads) k_refine_small(NaArgs a)
{
    __shared__ uint32_t s_count, s_err, s_nfail, s_done;
    const uint32_t n = a.n;
    uint32_t* col = reinterpret_cast<uint32_t*>(a.scratch + kNaCol);
    uint32_t* initlab = reinterpret_cast<uint32_t*>(a.scratch + kNaInit);
    unsigned long long* sig1 = reinterpret_cast<unsigned long long*>(a.scratch + kNaSig1);
    uint32_t* sig2 = reinterpret_cast<uint32_t*>(a.scratch + kNaSig2);
    uint32_t* slot = reinterpret_cast<uint32_t*>(a.scratch + kNaSlot);
    uint32_t* fail = reinterpret_cast<uint32_t*>(a.scratch + kNaFail);
    Entry* tab = reinterpret_cast<Entry*>(a.scratch + kNaTable);
    unsigned long long* cnt_all = reinterpret_cast<unsigned long long*>(a.scratch + kNaCount);
    uint32_t log2tab = 10;
    while (log2tab < kNaLog2Table && (1u << log2tab) < 2u * n) ++log2tab;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (n == 0) {
        if (threadIdx.x == 0) {
            a.result->blocks = 0;
            a.result->rounds = 0;
            a.result->repairs = 0;
            a.result->status = RBSC_OK;
        }
        return;
    }

    // The graph is checked before any read indexed by it: offsets[0] = 0,
    // offsets non-decreasing, offsets[n] = m (the stated arc count, at most
    // RBSC_NOALLOC_MAX_ARCS), every head < n.  Only then do col[idx[k]] and
    // cnt[col[idx[k]]] stay inside the scratch array.  A malformed graph ends
    // the call with RBSC_ERR_INVALID in d_result, nothing written to d_out.
    if (threadIdx.x == 0) s_err = 0;
    __syncthreads();
    for (uint32_t u = threadIdx.x; u <= n; u += kNaThreads) {
        const uint64_t o = na_off(a.off, a.off64, u);
        const bool bad = (u == 0 && o != 0ull) || (u == n && o != a.m) || (u < n && o > na_off(a.off, a.off64, u + 1));
        if (bad) s_err = 1;
    }
    __syncthreads();
    if (!*(volatile uint32_t*)&s_err)
        for (uint64_t k = threadIdx.x; k < a.m; k += kNaThreads)
            if (a.idx[k] >= n) s_err = 1;
    __syncthreads();
    if (*(volatile uint32_t*)&s_err) {
        if (threadIdx.x == 0) {
            a.result->blocks = 0;
            a.result->rounds = 0;
            a.result->repairs = 0;
            a.result->status = RBSC_ERR_INVALID;
        }
        return;
    }
    __syncthreads();

    // the scratch keeps the previous call's contents: clear what must start at zero
    if (threadIdx.x == 0) {
        s_err = 0;
        s_done = 0;
    }
    unsigned long long* cnt = cnt_all + (size_t)warp * kNaMaxNodes;
    for (uint32_t i = lane; i < n; i += 32) cnt[i] = 0ull;
    for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) {
        sig1[u] = 0ull;
        sig2[u] = 0u;
        fail[u] = 0u;
    }
    __syncthreads();

    // initial partition
    uint32_t prev;
    if (a.init) {
        prev = na_table_pass(1, n, col, a.init, sig1, sig2, fail, tab, log2tab, slot, a.seed, 0, &s_count, &s_err);
    } else {
        for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) col[u] = (n == 1u) ? kSingleton : 0u;
        prev = 1;
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) initlab[u] = col[u] & kLabelMask;
    __syncthreads();

    uint32_t round = 0, repairs = 0;
    int32_t status = RBSC_OK;
    for (;;) {
        // hashed rounds to the fixpoint
        for (;;) {
            if (round >= a.max_rounds) {
                status = RBSC_ERR_NOT_CONVERGED;
                break;
            }
            const uint64_t salt = pass_salt1(a.seed, round);
            for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) {
                if (col[u] & kSingleton) continue;
                const uint64_t b = na_off(a.off, a.off64, u), e = na_off(a.off, a.off64, u + 1);
                uint64_t s1 = 0;
                uint32_t s2 = 0;
                for (uint64_t k = b; k < e; ++k) {
                    uint64_t t1;
                    uint32_t t2;
                    arc_terms(col[a.idx[k]], salt, t1, t2);
                    if (a.wt) {
                        t1 *= a.wt[k];
                        t2 *= (uint32_t)a.wt[k];
                    }
                    s1 += t1;
                    s2 += t2;
                }
                sig1[u] = s1;
                sig2[u] = s2;
            }
            __syncthreads();
            const uint32_t blocks = na_table_pass(0, n, col, nullptr, sig1, sig2, fail, tab, log2tab, slot, a.seed,
                                                  a.hash_bits, &s_count, &s_err);
            ++round;
            const bool fixed = blocks == prev;
            prev = blocks;
            if (fixed) break;
        }
        if (status != RBSC_OK) break;
        // exact check: every node's (colour -> weight) multiset equals its block
        // representative's, counted in this warp's array over both rows
        if (threadIdx.x == 0) s_nfail = 0;
        __syncthreads();
        for (uint32_t u = warp; u < n; u += kNaWarps) {
            const uint32_t c = col[u];
            const uint32_t r = c & kLabelMask;
            if ((c & kSingleton) || r == u) continue;
            bool bad = initlab[u] != initlab[r];
            if (!bad) {
                const uint64_t bu = na_off(a.off, a.off64, u), eu = na_off(a.off, a.off64, u + 1);
                const uint64_t br = na_off(a.off, a.off64, r), er = na_off(a.off, a.off64, r + 1);
                for (uint64_t k = br + lane; k < er; k += 32)
                    atomicAdd(&cnt[col[a.idx[k]] & kLabelMask], (unsigned long long)(a.wt ? a.wt[k] : 1ull));
                for (uint64_t k = bu + lane; k < eu; k += 32)
                    atomicAdd(&cnt[col[a.idx[k]] & kLabelMask], (unsigned long long)(0ull - (a.wt ? a.wt[k] : 1ull)));
                __syncwarp();
                bool diff = false;
                for (uint64_t k = br + lane; k < er && !diff; k += 32) diff = cnt[col[a.idx[k]] & kLabelMask] != 0ull;
                for (uint64_t k = bu + lane; k < eu && !diff; k += 32) diff = cnt[col[a.idx[k]] & kLabelMask] != 0ull;
                bad = __any_sync(0xffffffffu, diff);
                __syncwarp();
                for (uint64_t k = br + lane; k < er; k += 32) cnt[col[a.idx[k]] & kLabelMask] = 0ull;
                for (uint64_t k = bu + lane; k < eu; k += 32) cnt[col[a.idx[k]] & kLabelMask] = 0ull;
                __syncwarp();
            }
            if (bad && lane == 0) {
                fail[u] = 1u;
                atomicAdd(&s_nfail, 1u);
            }
        }
        __syncthreads();
        if (*(volatile uint32_t*)&s_nfail == 0) break;
        // split the failing nodes from their blocks and refine again
        ++repairs;
        prev = na_table_pass(2, n, col, nullptr, sig1, sig2, fail, tab, log2tab, slot, a.seed, 0, &s_count, &s_err);
        for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) fail[u] = 0u;
        __syncthreads();
        if (repairs > n) {
            status = RBSC_ERR_DEVICE;
            break;
        }
    }
    if (s_err) status = RBSC_ERR_DEVICE;
    for (uint32_t u = threadIdx.x; u < n; u += kNaThreads) a.out[u] = col[u] & kLabelMask;
    if (threadIdx.x == 0) {
        a.result->blocks = prev;
        a.result->rounds = round;
        a.result->repairs = repairs;
        a.result->status = status;
    }
}

std::mutex g_na_mutex;
unsigned char* g_na_ptr[64] = {};

}  // namespace

rbsc_status rbsc_fail(rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...);

extern "C" rbsc_status rbsc_refine_noalloc(const rbsc_csr* g, const uint32_t* d_init_colors, uint32_t* d_out_labels,
                                           rbsc_noalloc_result* d_result, const rbsc_opts* opts, void* stream)
{
    if (!g || !d_out_labels || !d_result) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null argument");
    if (g->n > kNaMaxNodes)
        return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "rbsc_refine_noalloc: N = %u exceeds the limit of %u nodes", g->n,
                         kNaMaxNodes);
    if (g->m > RBSC_NOALLOC_MAX_ARCS)
        return rbsc_fail(nullptr, RBSC_ERR_TOO_LARGE, "rbsc_refine_noalloc: M = %llu exceeds the limit of %u arcs",
                         (unsigned long long)g->m, (unsigned)RBSC_NOALLOC_MAX_ARCS);
    if (g->offset_bytes != 4 && g->offset_bytes != 8) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "offset_bytes must be 4 or 8");
    if (!g->offsets || (g->m && !g->indices)) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null graph array");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return rbsc_fail(nullptr, RBSC_ERR_CUDA, "no current CUDA device");
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_ptr[dev]) {
            // once per device, with that device current: the device address of
            // the scratch array (its host-side name is not a device address)
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return rbsc_fail(nullptr, RBSC_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
            g_na_ptr[dev] = static_cast<unsigned char*>(p);
        }
        scratch = g_na_ptr[dev];
    }
    rbsc_opts o;
    if (opts) o = *opts;
    else rbsc_opts_default(&o);
    NaArgs a;
    a.n = g->n;
    a.m = g->m;
    a.off = g->offsets;
    a.off64 = g->offset_bytes == 8;
    a.idx = g->indices;
    a.wt = g->weights;
    a.init = d_init_colors;
    a.out = d_out_labels;
    a.result = d_result;
    a.scratch = scratch;
    a.seed = o.seed;
    a.max_rounds = o.max_rounds ? o.max_rounds : g->n + 1u;
    a.hash_bits = o.test_hash_bits < 0 ? 64u : (uint32_t)o.test_hash_bits;
    ++launch_counter();
    k_refine_small<<<1, kNaThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return rbsc_fail(nullptr, RBSC_ERR_CUDA, "k_refine_small launch failed: %s", cudaGetErrorString(e));
    return RBSC_OK;
}
