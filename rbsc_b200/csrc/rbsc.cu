// rbsc.cu -- host side of librbsc: contexts, resident graphs, the refinement
// driver (device-resident round loop in a CUDA graph with a while node), the
// exact check + repair, and the C ABI of include/rbsc.h.
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "common.cuh"
#include "prep_kernels.cuh"
#include "radix.cuh"
#include "refine_kernels.cuh"
#include "hot_kernels.cuh"
#include "scan.cuh"
#include "verify_kernels.cuh"
#include "internal.h"

using namespace rbsc;

namespace {
thread_local std::string g_global_error;
}

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
rbsc_status rbsc_fail(rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    else g_global_error = buf;
    return code;
}

rbsc_status rbsc_cuda_fail(rbsc_ctx* ctx, cudaError_t e, const char* what, int line)
{
    const rbsc_status code = (e == cudaErrorMemoryAllocation) ? RBSC_ERR_OOM : RBSC_ERR_CUDA;
    return rbsc_fail(ctx, code, "%s failed (line %d): %s (%d)", what, line, cudaGetErrorString(e), (int)e);
}

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return rbsc_cuda_fail(ctx, e_, #call, __LINE__); \
    } while (0)

#define CKS(call)                           \
    do {                                    \
        rbsc_status s_ = (call);            \
        if (s_ != RBSC_OK) return s_;       \
    } while (0)

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
// Block sizes: small requests in powers of two (at least 4 KB), large ones in
// whole 2 MB pages, so that a repeated request finds its block again.
static size_t pool_round(size_t bytes)
{
    if (bytes <= 4096) return 4096;
    if (bytes < (2u << 20)) {
        size_t b = 4096;
        while (b < bytes) b <<= 1;
        return b;
    }
    return (bytes + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
}

static void pool_raw_free(MemPool& p, void* b)
{
    if (p.pinned) cudaFreeHost(b);
    else cudaFree(b);
}

// Gives every unused block back to CUDA.
static void pool_release(MemPool& p)
{
    for (auto& kv : p.free_blocks) {
        p.sizes.erase(kv.second);
        pool_raw_free(p, kv.second);
    }
    p.free_blocks.clear();
    p.cached = 0;
}

static rbsc_status pool_alloc(rbsc_ctx* ctx, MemPool& p, void** out, size_t bytes)
{
    *out = nullptr;
    const size_t want = pool_round(bytes);
    // best fit among the unused blocks, if it wastes at most half
    auto it = p.free_blocks.lower_bound(want);
    if (it != p.free_blocks.end() && it->first <= 2 * want) {
        *out = it->second;
        p.cached -= it->first;
        p.free_blocks.erase(it);
        return RBSC_OK;
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        void* b = nullptr;
        const cudaError_t e = p.pinned ? cudaMallocHost(&b, want) : cudaMalloc(&b, want);
        if (e == cudaSuccess) {
            p.sizes[b] = want;
            *out = b;
            return RBSC_OK;
        }
        cudaGetLastError();
        if (attempt == 0 && p.cached) {
            pool_release(p);  // out of memory with blocks cached: give them back and retry
            continue;
        }
        return rbsc_fail(ctx, RBSC_ERR_OOM, "%s of %zu bytes failed: %s", p.pinned ? "cudaMallocHost" : "cudaMalloc", want,
                         cudaGetErrorString(e));
    }
    return RBSC_ERR_OOM;
}

static void pool_free(MemPool& p, void* b)
{
    auto it = p.sizes.find(b);
    if (it == p.sizes.end()) return;  // not ours (cannot happen)
    p.free_blocks.emplace(it->second, b);
    p.cached += it->second;
    // over the cap: drop the largest unused blocks
    while (p.cached > p.cap && !p.free_blocks.empty()) {
        auto last = std::prev(p.free_blocks.end());
        p.cached -= last->first;
        p.sizes.erase(last->second);
        pool_raw_free(p, last->second);
        p.free_blocks.erase(last);
    }
}

rbsc_status dev_alloc(rbsc_ctx* ctx, void** p, size_t bytes) { return pool_alloc(ctx, ctx->dpool, p, bytes); }

// Returns a block to the context's pool.  Work already queued on the
// context's stream that uses the block stays ordered before any later use,
// since every later user is queued on the same stream.
void dev_free(rbsc_ctx* ctx, void*& p)
{
    if (p) pool_free(ctx->dpool, p);
    p = nullptr;
}

rbsc_status host_alloc(rbsc_ctx* ctx, void** p, size_t bytes) { return pool_alloc(ctx, ctx->hpool, p, bytes); }

void host_free(rbsc_ctx* ctx, void*& p)
{
    if (p) pool_free(ctx->hpool, p);
    p = nullptr;
}

rbsc_status ensure_temp(rbsc_ctx* ctx, rbsc_graph* g, size_t bytes)
{
    if (g->tmp_bytes >= bytes) return RBSC_OK;
    dev_free(ctx, g->d_tmp);
    g->tmp_bytes = 0;
    CKS(dev_alloc(ctx, &g->d_tmp, bytes));
    g->tmp_bytes = bytes;
    return RBSC_OK;
}

static unsigned grid_for(uint64_t n, unsigned threads) { return (unsigned)std::max<uint64_t>(1, ceil_div<uint64_t>(n, threads)); }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" int32_t rbsc_abi_version(void) { return RBSC_ABI_VERSION; }

extern "C" void rbsc_opts_default(rbsc_opts* o)
{
    std::memset(o, 0, sizeof *o);
    o->relabel = RBSC_RELABEL_HASH;
    o->verify = 1;
    o->max_rounds = 0;
    o->use_graph = 1;
    o->seed = 0x5eed5eed12345678ull;
    o->test_hash_bits = 0;
}

extern "C" rbsc_ctx* rbsc_ctx_create(int32_t device, const rbsc_opts* opts)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        rbsc_fail(nullptr, RBSC_ERR_CUDA, "no CUDA device available: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if (device < 0 || device >= count) {
        rbsc_fail(nullptr, RBSC_ERR_INVALID, "device %d out of range (have %d)", device, count);
        return nullptr;
    }
    rbsc_ctx* ctx = new (std::nothrow) rbsc_ctx();
    if (!ctx) {
        rbsc_fail(nullptr, RBSC_ERR_OOM, "out of host memory");
        return nullptr;
    }
    ctx->device = device;
    if (opts) ctx->opts = *opts;
    else rbsc_opts_default(&ctx->opts);
    if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        rbsc_fail(nullptr, RBSC_ERR_CUDA, "context setup failed: %s", cudaGetErrorString(e));
        delete ctx;
        return nullptr;
    }
    for (auto& ev : ctx->ev) cudaEventCreate(&ev);
    for (auto& ev : ctx->ev_sig) cudaEventCreate(&ev);
    if ((e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming)) != cudaSuccess) {
        rbsc_fail(nullptr, RBSC_ERR_CUDA, "context setup failed: %s", cudaGetErrorString(e));
        rbsc_ctx_destroy(ctx);
        return nullptr;
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    return ctx;
}

extern "C" void rbsc_ctx_destroy(rbsc_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& ev : ctx->ev) cudaEventDestroy(ev);
    for (auto& ev : ctx->ev_sig) cudaEventDestroy(ev);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    cudaStreamDestroy(ctx->stream);
    pool_release(ctx->dpool);
    pool_release(ctx->hpool);
    delete ctx;
}

extern "C" void rbsc_ctx_trim(rbsc_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    pool_release(ctx->dpool);
    pool_release(ctx->hpool);
}

extern "C" const char* rbsc_last_error(const rbsc_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : g_global_error.c_str();
}

extern "C" rbsc_status rbsc_ctx_set_opts(rbsc_ctx* ctx, const rbsc_opts* opts)
{
    if (!ctx || !opts) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    ctx->opts = *opts;
    return RBSC_OK;
}

// ---------------------------------------------------------------------------
// resident graph
// ---------------------------------------------------------------------------
static void graph_release_refine(rbsc_graph* g)
{
    if (g->loop_exec) cudaGraphExecDestroy(g->loop_exec);
    if (g->loop_graph) cudaGraphDestroy(g->loop_graph);
    g->loop_exec = nullptr;
    g->loop_graph = nullptr;
    dev_free(g->ctx, (void*&)g->d_col[0]);
    dev_free(g->ctx, (void*&)g->d_as);
    dev_free(g->ctx, (void*&)g->d_gsync);
    dev_free(g->ctx, (void*&)g->d_pairs);
    dev_free(g->ctx, (void*&)g->d_grep);
    dev_free(g->ctx, (void*&)g->d_gcnt);
    for (int d = 0; d < 2; ++d) {
        dev_free(g->ctx, (void*&)g->cb.rows[d]);
        dev_free(g->ctx, (void*&)g->cb.off[d]);
        dev_free(g->ctx, (void*&)g->cb.src[d]);
        dev_free(g->ctx, (void*&)g->cb.idx[d]);
        dev_free(g->ctx, (void*&)g->cb.wt[d]);
        dev_free(g->ctx, (void*&)g->cb.head8[d]);
        dev_free(g->ctx, (void*&)g->cb.tile_row[d]);
        dev_free(g->ctx, (void*&)g->cb.split[d]);
        dev_free(g->ctx, (void*&)g->cb.nodes[d]);
        dev_free(g->ctx, (void*&)g->cb.chunk_row[d]);
    }
    dev_free(g->ctx, (void*&)g->d_initlab);
    dev_free(g->ctx, (void*&)g->d_sig);
    dev_free(g->ctx, (void*&)g->d_slot);
    dev_free(g->ctx, (void*&)g->d_joined);
    dev_free(g->ctx, (void*&)g->d_tab);
    dev_free(g->ctx, (void*&)g->d_tab8);
    dev_free(g->ctx, (void*&)g->d_srank);
    dev_free(g->ctx, (void*&)g->d_st);
    dev_free(g->ctx, (void*&)g->d_out);
    dev_free(g->ctx, (void*&)g->d_rank);
    dev_free(g->ctx, (void*&)g->d_hot_idx);
    dev_free(g->ctx, (void*&)g->d_hot_node);
    dev_free(g->ctx, (void*&)g->d_hot_rank);
    g->hot_state = 0;
    dev_free(g->ctx, (void*&)g->d_init);
    dev_free(g->ctx, (void*&)g->d_vflag);
    dev_free(g->ctx, (void*&)g->d_vrow);
    dev_free(g->ctx, (void*&)g->d_vl8);
    dev_free(g->ctx, (void*&)g->d_vl32);
    dev_free(g->ctx, (void*&)g->d_vllong);
    dev_free(g->ctx, (void*&)g->d_vdeg);
    dev_free(g->ctx, (void*&)g->d_vstart);
    dev_free(g->ctx, (void*&)g->d_fail);
    dev_free(g->ctx, (void*&)g->d_keys[0]);
    dev_free(g->ctx, (void*&)g->d_keys[1]);
    dev_free(g->ctx, (void*&)g->d_vals[0]);
    dev_free(g->ctx, (void*&)g->d_vals[1]);
    dev_free(g->ctx, (void*&)g->d_small);
    dev_free(g->ctx, g->d_tmp);
    g->tmp_bytes = 0;
    g->key_cap = 0;
    host_free(g->ctx, (void*&)g->h_st);
    host_free(g->ctx, (void*&)g->h_as);
    g->bufs = false;
    sortrelabel_release(g);
}

extern "C" void rbsc_graph_free(rbsc_graph* g)
{
    if (!g) return;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    // a refinement that stopped early may leave side-stream clears of its
    // buffers unjoined
    cudaStreamSynchronize(g->ctx->side);
    graph_release_refine(g);
    dev_free(g->ctx, (void*&)g->d_off);
    if (g->copy_stream) cudaStreamSynchronize(g->copy_stream);
    for (int i = 0; i < 2; ++i) {
        dev_free(g->ctx, (void*&)g->d_chunk[i]);
        dev_free(g->ctx, (void*&)g->d_chunk_wt[i]);
        if (g->ev_copied[i]) cudaEventDestroy(g->ev_copied[i]);
        if (g->ev_used[i]) cudaEventDestroy(g->ev_used[i]);
    }
    for (auto& ev : g->ev_chunk)
        if (ev) cudaEventDestroy(ev);
    if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
    if (g->host_arcs) {
        if (g->reg_idx) cudaHostUnregister(g->reg_idx);
        if (g->reg_wt) cudaHostUnregister(g->reg_wt);
        g->d_idx = nullptr;  // host memory of the caller
        g->d_wt = nullptr;
    }
    dev_free(g->ctx, (void*&)g->d_idx);
    dev_free(g->ctx, (void*&)g->d_wt);
    dev_free(g->ctx, (void*&)g->d_rows);
    dev_free(g->ctx, g->d_roff);
    dev_free(g->ctx, (void*&)g->d_tile_row);
    dev_free(g->ctx, (void*&)g->d_split);
    dev_free(g->ctx, (void*&)g->d_head8);
    delete g;
}

extern "C" rbsc_status rbsc_graph_info(const rbsc_graph* g, uint32_t* n, uint64_t* m)
{
    if (!g) return RBSC_ERR_INVALID;
    if (n) *n = g->n;
    if (m) *m = g->m;
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_graph_device_csr(const rbsc_graph* g, const uint64_t** d_offsets, const uint32_t** d_indices)
{
    if (!g) return RBSC_ERR_INVALID;
    if (d_offsets) *d_offsets = g->d_off;
    if (d_indices) *d_indices = g->d_idx;
    return RBSC_OK;
}

// Builds the tiling of a graph whose d_off / d_idx / d_wt are in place.
rbsc_status graph_prepare(rbsc_ctx* ctx, rbsc_graph* g)
{
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n;
    const uint64_t m = g->m;
    g->off32 = m < (1ull << 32);
    // validation (device-side, one error word)
    uint32_t* d_err = nullptr;
    CKS(dev_alloc(ctx, (void**)&d_err, sizeof(uint32_t) * 4));
    struct Guard { rbsc_ctx* c; uint32_t*& p; ~Guard() { dev_free(c, (void*&)p); } } guard{ctx, d_err};
    CK(cudaMemsetAsync(d_err, 0, sizeof(uint32_t) * 4, s));
    ++rbsc::launch_counter();
    k_validate<<<grid_for(std::max<uint64_t>(n, 1), 256) > 65535u * 16 ? 65535u * 16 : grid_for(std::max<uint64_t>(n, 1), 256), 256, 0, s>>>(
        n, m, g->d_off, g->stream_upload ? nullptr : g->d_idx, d_err);
    CK(cudaGetLastError());
    uint32_t herr = 0;
    CK(cudaMemcpyAsync(&herr, d_err, sizeof herr, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (herr & 3u) return rbsc_fail(ctx, RBSC_ERR_INVALID, "offsets are not a valid CSR (must start at 0, be non-decreasing and end at M)");
    if (herr & 4u) return rbsc_fail(ctx, RBSC_ERR_INVALID, "an arc head is >= N");

    // non-empty rows
    CKS(ensure_temp(ctx, g, scan_temp_bytes<uint32_t>((uint64_t)n + 1) + 1024));
    uint32_t* d_pos = nullptr;
    CKS(dev_alloc(ctx, (void**)&d_pos, sizeof(uint32_t) * ((size_t)n + 1)));
    struct Guard2 { rbsc_ctx* c; uint32_t*& p; ~Guard2() { dev_free(c, (void*&)p); } } guard2{ctx, d_pos};
    ++rbsc::launch_counter();
    k_nonempty_flags<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_off, d_pos);
    CK(cudaGetLastError());
    CK((exclusive_scan<uint32_t, uint32_t>(d_pos, d_pos, n, d_err + 1, g->d_tmp, s)));
    uint32_t K = 0;
    CK(cudaMemcpyAsync(&K, d_err + 1, sizeof K, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    g->K = K;
    CKS(dev_alloc(ctx, (void**)&g->d_rows, sizeof(uint32_t) * std::max<uint32_t>(K, 1)));
    CKS(dev_alloc(ctx, &g->d_roff, (g->off32 ? 4 : 8) * ((size_t)K + 1)));
    if (g->off32) {
        ++rbsc::launch_counter();
        k_prep_rows<uint32_t><<<grid_for(n, 256), 256, 0, s>>>(n, m, g->d_off, d_pos, K, g->d_rows, (uint32_t*)g->d_roff);
    }
    else {
        ++rbsc::launch_counter();
        k_prep_rows<uint64_t><<<grid_for(n, 256), 256, 0, s>>>(n, m, g->d_off, d_pos, K, g->d_rows, (uint64_t*)g->d_roff);
    }
    CK(cudaGetLastError());
    // tiles
    g->ntiles = (uint32_t)ceil_div<uint64_t>(m, kTileEdges);
    CKS(dev_alloc(ctx, (void**)&g->d_tile_row, sizeof(uint32_t) * ((size_t)g->ntiles + 1)));
    if (g->off32) {
        ++rbsc::launch_counter();
        k_tile_rows<uint32_t><<<grid_for((uint64_t)g->ntiles + 1, 256), 256, 0, s>>>(g->ntiles, K, (const uint32_t*)g->d_roff, g->d_tile_row);
    }
    else {
        ++rbsc::launch_counter();
        k_tile_rows<uint64_t><<<grid_for((uint64_t)g->ntiles + 1, 256), 256, 0, s>>>(g->ntiles, K, (const uint64_t*)g->d_roff, g->d_tile_row);
    }
    CK(cudaGetLastError());
    // row-head bitmap (one bit per arc, padded to whole tiles)
    {
        const size_t hbytes = ((size_t)g->ntiles * kTileEdges) / 8 + 16;
        CKS(dev_alloc(ctx, (void**)&g->d_head8, hbytes));
        CK(cudaMemsetAsync(g->d_head8, 0, hbytes, s));
        if (K > 0) {
            ++rbsc::launch_counter();
            if (g->off32)
                k_head_bits<uint32_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint32_t*)g->d_roff, (uint32_t*)g->d_head8);
            else
                k_head_bits<uint64_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint64_t*)g->d_roff, (uint32_t*)g->d_head8);
            CK(cudaGetLastError());
        }
    }
    // rows split across tiles
    if (K > 0) {
        CKS(ensure_temp(ctx, g, scan_temp_bytes<uint32_t>((uint64_t)K + 1) + 1024));
        uint32_t* d_sp = nullptr;
        CKS(dev_alloc(ctx, (void**)&d_sp, sizeof(uint32_t) * ((size_t)K + 1)));
        struct Guard3 { rbsc_ctx* c; uint32_t*& p; ~Guard3() { dev_free(c, (void*&)p); } } guard3{ctx, d_sp};
        if (g->off32) {
            ++rbsc::launch_counter();
            k_split_flags<uint32_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint32_t*)g->d_roff, d_sp);
        }
        else {
            ++rbsc::launch_counter();
            k_split_flags<uint64_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint64_t*)g->d_roff, d_sp);
        }
        CK(cudaGetLastError());
        CK((exclusive_scan<uint32_t, uint32_t>(d_sp, d_sp, K, d_err + 2, g->d_tmp, s)));
        uint32_t ns = 0;
        CK(cudaMemcpyAsync(&ns, d_err + 2, sizeof ns, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        g->nsplit = ns;
        CKS(dev_alloc(ctx, (void**)&g->d_split, sizeof(uint32_t) * std::max<uint32_t>(ns, 1)));
        if (g->off32) {
            ++rbsc::launch_counter();
            k_split_compact<uint32_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint32_t*)g->d_roff, g->d_rows, d_sp, g->d_split);
        }
        else {
            ++rbsc::launch_counter();
            k_split_compact<uint64_t><<<grid_for(K, 256), 256, 0, s>>>(K, (const uint64_t*)g->d_roff, g->d_rows, d_sp, g->d_split);
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
    } else {
        g->nsplit = 0;
        CKS(dev_alloc(ctx, (void**)&g->d_split, sizeof(uint32_t)));
    }
    return RBSC_OK;
}

static rbsc_status check_csr_args(rbsc_ctx* ctx, const rbsc_csr* c)
{
    if (!ctx) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null context");
    if (!c) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null graph");
    if (c->n >= 0x80000000u) return rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "N = %u: node ids must be < 2^31", c->n);
    if (c->offset_bytes != 4 && c->offset_bytes != 8) return rbsc_fail(ctx, RBSC_ERR_INVALID, "offset_bytes must be 4 or 8");
    if (c->offset_bytes == 4 && c->m >= (1ull << 32)) return rbsc_fail(ctx, RBSC_ERR_INVALID, "M >= 2^32 needs 8-byte offsets");
    if (!c->offsets) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null offsets");
    if (c->m > 0 && !c->indices) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null indices");
    return RBSC_OK;
}

// Allocates the CSR arrays of g (indices / weights padded to whole tiles).
rbsc_status graph_alloc_csr(rbsc_ctx* ctx, rbsc_graph* g, bool weighted)
{
    const uint64_t padded = ceil_div<uint64_t>(std::max<uint64_t>(g->m, 1), kTileEdges) * kTileEdges;
    g->weighted = weighted;
    CKS(dev_alloc(ctx, (void**)&g->d_off, sizeof(uint64_t) * ((size_t)g->n + 1)));
    CKS(dev_alloc(ctx, (void**)&g->d_idx, sizeof(uint32_t) * padded));
    if (padded > g->m) CK(cudaMemsetAsync(g->d_idx + g->m, 0, sizeof(uint32_t) * (padded - g->m), ctx->stream));
    if (weighted) {
        CKS(dev_alloc(ctx, (void**)&g->d_wt, sizeof(uint64_t) * padded));
        if (padded > g->m) CK(cudaMemsetAsync(g->d_wt + g->m, 0, sizeof(uint64_t) * (padded - g->m), ctx->stream));
    }
    return RBSC_OK;
}

// defer_heads: the heads are not copied here; they arrive in chunks during
// the first pass that reads them (stream_signature's upload mode), which
// overlaps their copy with the initial colours, the setup and that pass.
static rbsc_status graph_load(rbsc_ctx* ctx, const rbsc_csr* c, bool from_device, rbsc_graph** out, double* h2d_ms,
                              uint64_t* h2d_bytes, bool defer_heads = false, const uint32_t* h_init = nullptr)
{
    *out = nullptr;
    CKS(check_csr_args(ctx, c));
    CK(cudaSetDevice(ctx->device));
    rbsc_graph* g = new (std::nothrow) rbsc_graph();
    if (!g) return rbsc_fail(ctx, RBSC_ERR_OOM, "out of host memory");
    g->ctx = ctx;
    g->n = c->n;
    g->m = c->m;
    rbsc_status st = graph_alloc_csr(ctx, g, c->weights != nullptr);
    if (st != RBSC_OK) {
        rbsc_graph_free(g);
        return st;
    }
    cudaStream_t s = ctx->stream;
    const cudaMemcpyKind kind = from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaSuccess;
    const size_t offb = (size_t)c->offset_bytes * ((size_t)c->n + 1);
    uint64_t bytes = offb + sizeof(uint32_t) * c->m + (c->weights ? sizeof(uint64_t) * c->m : 0);
    if (c->offset_bytes == 8) {
        e = cudaMemcpyAsync(g->d_off, c->offsets, offb, kind, s);
    } else {
        // stage the 32-bit offsets in the (not yet used) index buffer tail? use a scratch buffer
        void* tmp = nullptr;
        st = dev_alloc(ctx, &tmp, offb);
        if (st != RBSC_OK) {
            rbsc_graph_free(g);
            return st;
        }
        e = cudaMemcpyAsync(tmp, c->offsets, offb, kind, s);
        if (e == cudaSuccess) {
            ++rbsc::launch_counter();
            k_widen_offsets<uint32_t><<<grid_for((uint64_t)c->n + 1, 256), 256, 0, s>>>((uint64_t)c->n + 1, (const uint32_t*)tmp, g->d_off);
            e = cudaGetLastError();
        }
        cudaStreamSynchronize(s);
        dev_free(ctx, tmp);
    }
    defer_heads = defer_heads && !from_device && !c->weights && c->m > 0;
    // the one-shot call's initial colours: copied right behind the offsets,
    // ahead of the heads, whose early copies (below) would otherwise hold
    // them back on the host link
    if (e == cudaSuccess && defer_heads && h_init && c->n) {
        st = dev_alloc(ctx, (void**)&g->d_init, 4 * (size_t)c->n);
        if (st != RBSC_OK) {
            rbsc_graph_free(g);
            return st;
        }
        e = cudaMemcpyAsync(g->d_init, h_init, 4 * (size_t)c->n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) g->h_init_loaded = h_init;
    }
    if (defer_heads) {
        g->stream_upload = true;
        g->h_upload = c->indices;
        g->chunk_tiles = (uint32_t)std::max<uint64_t>(1, ceil_div<uint64_t>(ceil_div<uint64_t>(c->m, kTileEdges), 8));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&g->ev_copied[i], cudaEventDisableTiming);
        // a page-locked source: issue every chunk's copy now, behind the
        // offsets (a pageable one is copied chunk by chunk in the first pass:
        // its copies would hold the host here)
        cudaPointerAttributes pa{};
        const cudaError_t qe = e == cudaSuccess ? cudaPointerGetAttributes(&pa, c->indices) : cudaSuccess;
        if (qe != cudaSuccess) cudaGetLastError();  // not a pointer CUDA knows: no early copies
        const uint64_t nt = ceil_div<uint64_t>(c->m, kTileEdges);
        if (e == cudaSuccess && qe == cudaSuccess && pa.type == cudaMemoryTypeHost &&
            ceil_div<uint64_t>(nt, g->chunk_tiles) <= (uint64_t)rbsc_graph::kUploadChunks) {
            int k = 0;
            for (uint64_t t = 0; t < nt && e == cudaSuccess; t += g->chunk_tiles, ++k) {
                const uint64_t a0 = t * kTileEdges, a1 = std::min<uint64_t>(c->m, (t + g->chunk_tiles) * kTileEdges);
                e = cudaEventCreateWithFlags(&g->ev_chunk[k], cudaEventDisableTiming);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(g->d_idx + a0, c->indices + a0, 4 * (a1 - a0), cudaMemcpyHostToDevice, g->copy_stream);
                if (e == cudaSuccess) e = cudaEventRecord(g->ev_chunk[k], g->copy_stream);
            }
            g->upload_issued = e == cudaSuccess;
        }
    } else if (e == cudaSuccess && c->m) {
        e = cudaMemcpyAsync(g->d_idx, c->indices, sizeof(uint32_t) * c->m, kind, s);
    }
    if (e == cudaSuccess && c->weights && c->m) e = cudaMemcpyAsync(g->d_wt, c->weights, sizeof(uint64_t) * c->m, kind, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    auto t1 = std::chrono::steady_clock::now();
    if (h2d_ms) *h2d_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (h2d_bytes) *h2d_bytes = from_device ? 0 : bytes;
    if (e != cudaSuccess) {
        rbsc_cuda_fail(ctx, e, "graph copy", __LINE__);
        rbsc_graph_free(g);
        return e == cudaErrorMemoryAllocation ? RBSC_ERR_OOM : RBSC_ERR_CUDA;
    }
    st = graph_prepare(ctx, g);
    if (st != RBSC_OK) {
        rbsc_graph_free(g);
        return st;
    }
    *out = g;
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_graph_upload(rbsc_ctx* ctx, const rbsc_csr* host_graph, rbsc_graph** out)
{
    if (!out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null output");
    return graph_load(ctx, host_graph, false, out, nullptr, nullptr);
}

extern "C" rbsc_status rbsc_graph_from_device(rbsc_ctx* ctx, const rbsc_csr* device_graph, rbsc_graph** out)
{
    if (!out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null output");
    return graph_load(ctx, device_graph, true, out, nullptr, nullptr);
}

// Device-accessible view of a host array: page-locked memory is used as it
// is; pageable memory is registered (mapped, read-only) and *reg records it.
static rbsc_status map_host(rbsc_ctx* ctx, const void* p, size_t bytes, void** dev, void** reg)
{
    *dev = nullptr;
    *reg = nullptr;
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        at.type = cudaMemoryTypeUnregistered;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged)
        return rbsc_fail(ctx, RBSC_ERR_INVALID, "streamed graph: arcs must be in host memory");
    if (at.type != cudaMemoryTypeHost) {
        e = cudaHostRegister(const_cast<void*>(p), bytes, cudaHostRegisterMapped | cudaHostRegisterReadOnly);
        if (e != cudaSuccess) return rbsc_cuda_fail(ctx, e, "cudaHostRegister", __LINE__);
        *reg = const_cast<void*>(p);
    }
    e = cudaHostGetDevicePointer(dev, const_cast<void*>(p), 0);
    if (e != cudaSuccess) {
        if (*reg) cudaHostUnregister(*reg);
        *reg = nullptr;
        return rbsc_cuda_fail(ctx, e, "cudaHostGetDevicePointer", __LINE__);
    }
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_graph_upload_streamed(rbsc_ctx* ctx, const rbsc_csr* c, uint64_t batch_arcs, uint64_t resident_arcs,
                                                  rbsc_graph** out)
{
    if (!out) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null output");
    *out = nullptr;
    CKS(check_csr_args(ctx, c));
    CK(cudaSetDevice(ctx->device));
    rbsc_graph* g = new (std::nothrow) rbsc_graph();
    if (!g) return rbsc_fail(ctx, RBSC_ERR_OOM, "out of host memory");
    struct Guard { rbsc_graph*& g; ~Guard() { if (g) rbsc_graph_free(g); } } guard{g};
    g->ctx = ctx;
    g->n = c->n;
    g->m = c->m;
    g->weighted = c->weights != nullptr;
    g->host_arcs = true;
    g->arcs_on_host = true;
    cudaStream_t s = ctx->stream;
    if (c->m) {
        void* dv = nullptr;
        CKS(map_host(ctx, c->indices, 4 * (size_t)c->m, &dv, &g->reg_idx));
        g->d_idx = static_cast<uint32_t*>(dv);
        if (c->weights) {
            CKS(map_host(ctx, c->weights, 8 * (size_t)c->m, &dv, &g->reg_wt));
            g->d_wt = static_cast<uint64_t*>(dv);
        }
    }
    // offsets in device memory (widened to 64 bits)
    CKS(dev_alloc(ctx, (void**)&g->d_off, sizeof(uint64_t) * ((size_t)g->n + 1)));
    const size_t offb = (size_t)c->offset_bytes * ((size_t)c->n + 1);
    if (c->offset_bytes == 8) {
        CK(cudaMemcpyAsync(g->d_off, c->offsets, offb, cudaMemcpyHostToDevice, s));
    } else {
        void* tmp = nullptr;
        CKS(dev_alloc(ctx, &tmp, offb));
        cudaError_t e = cudaMemcpyAsync(tmp, c->offsets, offb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            ++rbsc::launch_counter();
            k_widen_offsets<uint32_t><<<grid_for((uint64_t)c->n + 1, 256), 256, 0, s>>>((uint64_t)c->n + 1, (const uint32_t*)tmp, g->d_off);
            e = cudaGetLastError();
        }
        cudaStreamSynchronize(s);
        dev_free(ctx, tmp);
        if (e != cudaSuccess) return rbsc_cuda_fail(ctx, e, "offsets", __LINE__);
    }
    CK(cudaStreamSynchronize(s));
    CKS(graph_prepare(ctx, g));  // validates the heads (read from host memory)
    const uint64_t batch = batch_arcs ? batch_arcs : std::max<uint64_t>(1, ceil_div<uint64_t>(c->m, 4));
    g->chunk_tiles = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(batch, kTileEdges), std::max<uint32_t>(g->ntiles, 1)));
    g->resident_cap = resident_arcs ? resident_arcs : std::min<uint64_t>(std::max<uint64_t>(c->m, 1), 1ull << 31);
    const size_t chunk = (size_t)g->chunk_tiles * kTileEdges;
    for (int i = 0; i < 2; ++i) {
        CKS(dev_alloc(ctx, (void**)&g->d_chunk[i], 4 * chunk));
        if (g->weighted) CKS(dev_alloc(ctx, (void**)&g->d_chunk_wt[i], 8 * chunk));
        CK(cudaEventCreateWithFlags(&g->ev_copied[i], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&g->ev_used[i], cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
    *out = g;
    g = nullptr;
    return RBSC_OK;
}

// ---------------------------------------------------------------------------
// refinement
// ---------------------------------------------------------------------------
static uint32_t log2_ceil(uint64_t x)
{
    uint32_t r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}

static rbsc_status ensure_refine_bufs(rbsc_ctx* ctx, rbsc_graph* g)
{
    if (g->bufs) return RBSC_OK;
    const size_t n = std::max<uint32_t>(g->n, 1);
    CKS(dev_alloc(ctx, (void**)&g->d_col[0], 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_initlab, 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_sig, sizeof(Sig) * n));
    CKS(dev_alloc(ctx, (void**)&g->d_slot, 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_joined, 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_out, 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_rank, 2 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_small, 256));
    g->log2tab = std::max<uint32_t>(10, log2_ceil(2ull * n));
    CKS(dev_alloc(ctx, (void**)&g->d_tab, sizeof(Entry) << g->log2tab));
    CKS(dev_alloc(ctx, (void**)&g->d_tab8, sizeof(unsigned long long) << g->log2tab));
    CKS(dev_alloc(ctx, (void**)&g->d_srank, (size_t)4 << g->log2tab));
    CKS(dev_alloc(ctx, (void**)&g->d_st, sizeof(RoundState)));
    CKS(host_alloc(ctx, (void**)&g->h_st, sizeof(RoundState)));
    CKS(host_alloc(ctx, (void**)&g->h_as, sizeof(ActiveSet)));
    // active set: node lists, followers, group representatives, compacted arc sets
    CKS(dev_alloc(ctx, (void**)&g->d_as, sizeof(ActiveSet)));
    CKS(dev_alloc(ctx, (void**)&g->d_gsync, sizeof(GridSync)));
    CKS(dev_alloc(ctx, (void**)&g->d_pairs, 8 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_grep, 4 * n));
    CKS(dev_alloc(ctx, (void**)&g->d_gcnt, 4 * n));
    g->compact_arcs = g->m > 0;
    const size_t K = std::max<uint32_t>(g->K, 1);
    // compacted arc sets: as large as the graph's own (in device memory), or
    // the resident capacity of a streamed graph; k_compact_decide copies only
    // what fits (and what fits 32-bit offsets)
    const size_t cap = g->host_arcs ? (size_t)std::max<uint64_t>(g->resident_cap, 1)
                                    : (size_t)std::max<uint64_t>(ceil_div<uint64_t>(3 * g->m, 4), 1);
    const size_t ctiles = ceil_div<uint64_t>(std::min<uint64_t>(cap, 0xffffffffull), kTileEdges);
    const size_t cpad = ctiles * kTileEdges;
    for (int d = 0; d < 2; ++d) {
        CKS(dev_alloc(ctx, (void**)&g->cb.nodes[d], 4 * n));
        if (!g->compact_arcs) continue;
        CKS(dev_alloc(ctx, (void**)&g->cb.rows[d], 4 * K));
        CKS(dev_alloc(ctx, (void**)&g->cb.off[d], 4 * (K + 1)));
        CKS(dev_alloc(ctx, (void**)&g->cb.src[d], 8 * K));
        CKS(dev_alloc(ctx, (void**)&g->cb.idx[d], 4 * cpad));
        if (g->weighted) CKS(dev_alloc(ctx, (void**)&g->cb.wt[d], 8 * cpad));
        CKS(dev_alloc(ctx, (void**)&g->cb.head8[d], cpad / 8 + 16));
        CKS(dev_alloc(ctx, (void**)&g->cb.tile_row[d], 4 * (ctiles + 1)));
        CKS(dev_alloc(ctx, (void**)&g->cb.split[d], 4 * (ctiles + 1)));
        CKS(dev_alloc(ctx, (void**)&g->cb.chunk_row[d], 4 * (cpad / 16 + 1)));
    }
    CK(cudaMemsetAsync(g->d_sig, 0, sizeof(Sig) * n, ctx->stream));
    CK(cudaMemsetAsync(g->d_tab, 0, sizeof(Entry) << g->log2tab, ctx->stream));
    g->next_stamp = 1;
    g->bufs = true;
    return RBSC_OK;
}

// Hot heads of the first pass (hot_kernels.cuh): for a resident graph with
// >= 2^22 arcs in device memory, unless the options choose another
// signature kernel.
static uint32_t hot_limit_log2(const rbsc_ctx* ctx)
{
    const int32_t l = ctx->opts.hot_log2;
    if (l == 0) return kHotMaxLog2;
    return (uint32_t)std::min<int32_t>(std::max<int32_t>(l, (int32_t)kHotMinLog2), (int32_t)kHotMaxLog2);
}

static bool hot_wanted(const rbsc_ctx* ctx, const rbsc_graph* g)
{
    const int32_t k = ctx->opts.sig_kernel;
    return (k == 0 || k == 3 || k == 4) && !g->host_arcs && !g->oneshot && !g->stream_upload && g->m >= (1ull << 22) && g->n > 1;
}

// In-degree threshold that at most `limit` nodes reach, from the binned
// in-degrees (in-degree >= 2 only); 0 when no node qualifies.
static uint32_t hot_threshold(const uint32_t* bins, uint64_t limit)
{
    uint64_t above = 0;
    uint32_t thr = 0;
    for (uint32_t b = kHotBins; b-- > 2;) {
        if (above + bins[b] > limit) break;
        above += bins[b];
        if (above) thr = hot_bin_floor(b);
    }
    return thr;
}

// cuTensorMapEncodeTiled from the driver, looked up once (the library links
// the runtime statically, not libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                  const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// The hot-head copy as a tensor for k_signature_hot_tma: 32 heads (128 B) a
// row, mpad / 32 rows, boxes of 16 rows (one 512-arc tile), 128-byte
// swizzle.  Tile t is the box at row 16 t, an int32 coordinate.
static bool encode_hot_tmap(rbsc_graph* g)
{
    g->hot_tma = false;
    const EncodeTiledFn enc = encode_tiled();
    const uint64_t rows = (uint64_t)g->ntiles * (kTileEdges / 32);
    g->hot_tma_err = !enc ? -1 : -2;
    if (!enc || !g->d_hot_idx || rows == 0 || rows >= (1ull << 31)) return false;
    const cuuint64_t dims[2] = {32, rows};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {32, kTileEdges / 32};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(&g->hot_tmap, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, g->d_hot_idx, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    g->hot_tma = r == CUDA_SUCCESS;
    g->hot_tma_err = (int)r;
    return g->hot_tma;
}

// Dynamic shared memory of k_signature_hot_tma: the staged table, 1 KB of
// alignment slack, one 2 KB buffer per warp.
static size_t hot_tma_smem(uint32_t hot_bytes) { return (size_t)hot_bytes + 1024 + (kHotThreads / 32) * kTmaTileBytes; }

// Builds the hot heads of a graph once per size limit: in-degrees, the
// threshold, the slots, the encoded copy of the heads.  false (nothing kept)
// when no node qualifies or device memory is short: the plain kernel runs.
// The tensor map of the copy is made here too (k_signature_hot_tma).
static rbsc_status build_hot(rbsc_ctx* ctx, rbsc_graph* g, bool* ready)
{
    const uint32_t lim = hot_limit_log2(ctx);
    *ready = false;
    if (g->hot_state != 0 && g->hot_log2 == lim) {
        *ready = g->hot_state > 0;
        return RBSC_OK;
    }
    cudaStream_t s = ctx->stream;
    dev_free(ctx, (void*&)g->d_hot_idx);
    dev_free(ctx, (void*&)g->d_hot_node);
    dev_free(ctx, (void*&)g->d_hot_rank);
    g->hot_state = -1;
    g->hot_log2 = lim;
    g->hot_n = g->hot_bytes = 0;
    const uint32_t n = g->n;
    const uint64_t mpad = (uint64_t)g->ntiles * kTileEdges;
    uint32_t* deg = nullptr;
    uint32_t* slot = nullptr;
    uint32_t* bins = nullptr;
    void* tmp = nullptr;
    auto drop = [&]() {
        dev_free(ctx, (void*&)deg);
        dev_free(ctx, (void*&)slot);
        dev_free(ctx, (void*&)bins);
        dev_free(ctx, tmp);
    };
    const size_t tbytes = scan_temp_bytes<uint32_t>((uint64_t)n) + 256;
    if (dev_alloc(ctx, (void**)&deg, 4ull * n) != RBSC_OK || dev_alloc(ctx, (void**)&slot, 4ull * n + 16) != RBSC_OK ||
        dev_alloc(ctx, (void**)&bins, 4 * kHotBins) != RBSC_OK || dev_alloc(ctx, &tmp, tbytes) != RBSC_OK) {
        drop();
        return RBSC_OK;
    }
    const unsigned agrid = (unsigned)ctx->sm_count * 16;
    CK(cudaMemsetAsync(deg, 0, 4ull * n, s));
    CK(cudaMemsetAsync(bins, 0, 4 * kHotBins, s));
    ++rbsc::launch_counter();
    k_hot_indeg<<<agrid, 256, 0, s>>>(g->d_idx, g->m, deg);
    ++rbsc::launch_counter();
    k_hot_hist<<<(unsigned)ctx->sm_count * 4, 256, 0, s>>>(n, deg, bins);
    CK(cudaGetLastError());
    uint32_t hb[kHotBins];
    CK(cudaMemcpyAsync(hb, bins, sizeof hb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint32_t thr = hot_threshold(hb, 1ull << lim);
    if (thr < 2) {
        drop();
        return RBSC_OK;
    }
    ++rbsc::launch_counter();
    k_hot_flags<<<grid_for(n, 256), 256, 0, s>>>(n, deg, thr);
    uint32_t* total = slot + n;
    CK((exclusive_scan<uint32_t, uint32_t>(deg, slot, n, total, tmp, s)));
    uint32_t hot_n = 0;
    CK(cudaMemcpyAsync(&hot_n, total, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint32_t hot_bytes = (uint32_t)ceil_div<uint64_t>(hot_n, 16) * 16;
    if (hot_n == 0 || hot_n > (1u << lim) || dev_alloc(ctx, (void**)&g->d_hot_node, 4ull * hot_n) != RBSC_OK ||
        dev_alloc(ctx, (void**)&g->d_hot_rank, hot_bytes) != RBSC_OK || dev_alloc(ctx, (void**)&g->d_hot_idx, 4 * mpad) != RBSC_OK) {
        dev_free(ctx, (void*&)g->d_hot_node);
        dev_free(ctx, (void*&)g->d_hot_rank);
        drop();
        return RBSC_OK;
    }
    ++rbsc::launch_counter();
    k_hot_assign<<<grid_for(n, 256), 256, 0, s>>>(n, deg, slot, g->d_hot_node);
    ++rbsc::launch_counter();
    k_hot_encode<<<agrid, 256, 0, s>>>(g->d_idx, g->m, deg, g->d_hot_idx);
    CK(cudaGetLastError());
    CK(cudaFuncSetAttribute(k_signature_hot<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 1 << kHotMaxLog2));
    CK(cudaFuncSetAttribute(k_signature_hot<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 1 << kHotMaxLog2));
    if (encode_hot_tmap(g)) {
        const int smax = (int)hot_tma_smem(1u << kHotMaxLog2);
        if (cudaFuncSetAttribute(k_signature_hot_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess ||
            cudaFuncSetAttribute(k_signature_hot_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess) {
            cudaGetLastError();
            g->hot_tma = false;
            g->hot_tma_err = -3;
        }
    }
    CK(cudaStreamSynchronize(s));
    drop();
    g->hot_n = hot_n;
    g->hot_bytes = hot_bytes;
    g->hot_state = 1;
    *ready = true;
    return RBSC_OK;
}

// The persistent kernel takes over once both the active arcs and the listed
// nodes are at most 2^persist_log2 (option; default 22).
static uint64_t persist_limit(const rbsc_ctx* ctx)
{
    const int32_t l = ctx->opts.persist_log2;
    if (l < 0) return 0;
    return 1ull << (l == 0 ? 22 : std::min(l, 31));
}

// Grids of the pass kernels: one thread (or warp) per unit of work, at most
// grid_per_sm blocks per SM (option; default 16), striding beyond.
static unsigned persistent_grid(rbsc_ctx* ctx, uint64_t work, unsigned per_block)
{
    const uint64_t per_sm = ctx->opts.grid_per_sm > 0 ? (uint64_t)ctx->opts.grid_per_sm : 16ull;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(work, per_block), (uint64_t)ctx->sm_count * per_sm));
}

// CUDA events around the kernels of one pass (profiling only).
struct PassTimer {
    cudaEvent_t ev[6];
};

// Launches the kernels of one hashed pass on stream s (also used for capture).
// First-pass gather variants (see k_signature / k_signature_uniform).
enum FirstPass { kPassFull = 0, kPassUniform = 1, kPassRank8 = 2, kPassRank16 = 3 };

// The signature kernel with tiles staged in shared memory by bulk copies
// (k_signature_staged): unweighted arc sets, when the options ask for it.
static bool staged_signature(const rbsc_ctx* ctx, const rbsc_graph* g)
{
    return !g->weighted && ctx->opts.sig_kernel == 2;
}

template <typename ColT>
static void launch_signature_chunk(bool weighted, bool staged, unsigned grid, cudaStream_t s, ActiveSet* as, RoundState* st,
                                   const ColT* col, Sig* sig, TileRange r)
{
    ++rbsc::launch_counter();
    if (staged && !weighted) k_signature_staged<ColT><<<grid, kTileThreads, 0, s>>>(as, st, col, sig, r, 1);
    else if (weighted) k_signature_chunk<true, ColT><<<grid, kTileThreads, 0, s>>>(as, st, col, sig, r);
    else k_signature_chunk<false, ColT><<<grid, kTileThreads, 0, s>>>(as, st, col, sig, r);
}

// The signature kernel over arcs in host memory: chunks of chunk_tiles tiles
// are copied into two device buffers on copy_stream; chunk c's copy waits
// until the kernel that read its buffer (chunk c-2) is done, and its kernel
// waits for the copy, so copies run beside the kernels of earlier chunks.
//
// Upload mode (g->stream_upload, the one-shot refinement of an unweighted
// graph): the chunks go straight to their final place in d_idx, each checked
// by k_validate_heads before its signature kernel reads it; after the pass
// the arcs are resident.
static rbsc_status stream_signature(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s, int first)
{
    const uint64_t m = g->m;
    const uint32_t ntiles = g->ntiles;
    const bool upload = g->stream_upload;
    for (uint32_t t0 = 0, c = 0; t0 < ntiles; t0 += g->chunk_tiles, ++c) {
        const uint32_t t1 = (uint32_t)std::min<uint64_t>(ntiles, (uint64_t)t0 + g->chunk_tiles);
        const uint64_t a0 = (uint64_t)t0 * kTileEdges, a1 = std::min<uint64_t>(m, (uint64_t)t1 * kTileEdges);
        const int slot = (int)(c & 1u);
        if (upload && g->upload_issued) {
            // copied since the load (the same chunks, in order)
            CK(cudaStreamWaitEvent(s, g->ev_chunk[c], 0));
        } else {
            if (upload) {
                CK(cudaMemcpyAsync(g->d_idx + a0, g->h_upload + a0, 4 * (a1 - a0), cudaMemcpyHostToDevice, g->copy_stream));
            } else {
                CK(cudaStreamWaitEvent(g->copy_stream, g->ev_used[slot], 0));
                CK(cudaMemcpyAsync(g->d_chunk[slot], g->d_idx + a0, 4 * (a1 - a0), cudaMemcpyHostToDevice, g->copy_stream));
                if (g->weighted)
                    CK(cudaMemcpyAsync(g->d_chunk_wt[slot], g->d_wt + a0, 8 * (a1 - a0), cudaMemcpyHostToDevice, g->copy_stream));
            }
            CK(cudaEventRecord(g->ev_copied[slot], g->copy_stream));
            CK(cudaStreamWaitEvent(s, g->ev_copied[slot], 0));
        }
        if (upload) {
            ++rbsc::launch_counter();
            k_validate_heads<<<persistent_grid(ctx, ceil_div<uint64_t>(a1 - a0, 256), 1), 256, 0, s>>>(a0, a1, g->n, g->d_idx,
                                                                                                      g->d_st);
            CK(cudaGetLastError());
        }
        const TileRange r = upload ? TileRange{t0, t1, g->d_idx + a0, nullptr, a0}
                                   : TileRange{t0, t1, g->d_chunk[slot], g->weighted ? g->d_chunk_wt[slot] : nullptr, a0};
        const unsigned grid = persistent_grid(ctx, t1 - t0, kTileThreads / 32);
        const bool st = staged_signature(ctx, g);
        if (first == kPassRank8)
            launch_signature_chunk<uint8_t>(g->weighted, st, grid, s, g->d_as, g->d_st,
                                            reinterpret_cast<const uint8_t*>(g->d_rank), g->d_sig, r);
        else if (first == kPassRank16)
            launch_signature_chunk<uint16_t>(g->weighted, st, grid, s, g->d_as, g->d_st,
                                             reinterpret_cast<const uint16_t*>(g->d_rank), g->d_sig, r);
        else
            launch_signature_chunk<uint32_t>(g->weighted, st, grid, s, g->d_as, g->d_st, g->d_col[0], g->d_sig, r);
        CK(cudaGetLastError());
        if (!upload) CK(cudaEventRecord(g->ev_used[slot], s));
        g->streamed_bytes += (a1 - a0) * (g->weighted ? 12 : 4);
    }
    ++g->streamed_passes;
    g->stream_upload = false;
    return RBSC_OK;
}

// An upload still pending when a pass that reads no arcs (the uniform first
// pass) would be followed by kernels that do: copy and check the rest now.
static rbsc_status finish_upload(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s)
{
    if (g->m) {
        if (g->upload_issued) {
            // the chunks were copied in order on copy_stream: the last one's
            // event covers them all
            int last = rbsc_graph::kUploadChunks - 1;
            while (last > 0 && !g->ev_chunk[last]) --last;
            CK(cudaStreamWaitEvent(s, g->ev_chunk[last], 0));
        } else {
            CK(cudaMemcpyAsync(g->d_idx, g->h_upload, 4 * g->m, cudaMemcpyHostToDevice, s));
        }
        ++rbsc::launch_counter();
        k_validate_heads<<<persistent_grid(ctx, ceil_div<uint64_t>(g->m, 256), 1), 256, 0, s>>>(0, g->m, g->n, g->d_idx, g->d_st);
        CK(cudaGetLastError());
    }
    g->stream_upload = false;
    return RBSC_OK;
}

static rbsc_status launch_pass(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s, cudaGraphConditionalHandle h, int use_handle,
                               PassTimer* t = nullptr, int first = kPassFull, uint32_t c0 = 0)
{
    const uint32_t n = g->n;
    const unsigned clear_grid = (unsigned)std::min<uint64_t>(ctx->sm_count * 8ull, grid_for(1ull << g->log2tab, 256));
    const unsigned ngrid = persistent_grid(ctx, n, kNodeThreads);
    const bool hash = ctx->opts.relabel != RBSC_RELABEL_SORT;
    if (t) CK(cudaEventRecord(t->ev[0], s));
    ++rbsc::launch_counter();
    k_clear_table<<<clear_grid, 256, 0, s>>>(g->d_st, g->d_tab, 1ull << g->log2tab);
    if (hash) {
        // the list table's window, zeroed on the side stream beside the
        // signature kernel (which neither reads nor writes the table); the
        // inserts wait for it below
        CK(cudaEventRecord(ctx->ev_fork, s));
        CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
        ++rbsc::launch_counter();
        k_clear_window8<<<clear_grid, 256, 0, ctx->side>>>(g->d_as, g->d_tab8, g->log2tab);
        CK(cudaEventRecord(ctx->ev_join, ctx->side));
    }
    if (t) CK(cudaEventRecord(t->ev[1], s));
    // the host-launched first pass is never captured: time its signature kernel
    if (first != kPassFull) CK(cudaEventRecord(ctx->ev_sig[0], s));
    const bool streamed = (g->arcs_on_host || g->stream_upload) && g->m > 0 && first != kPassUniform;
    if (g->stream_upload && !streamed) CKS(finish_upload(ctx, g, s));
    if (streamed) {
        CKS(stream_signature(ctx, g, s, first));
    } else if (g->m > 0) {
        const unsigned blocks = persistent_grid(ctx, g->ntiles, kTileThreads / 32);
        ++rbsc::launch_counter();
        if (first == kPassUniform) {
            const unsigned ugrid = persistent_grid(ctx, g->K, kNodeThreads);
            if (g->weighted)
                k_signature_uniform<true><<<ugrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_off, g->d_wt, c0, g->d_sig);
            else
                k_signature_uniform<false><<<ugrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_off, g->d_wt, c0, g->d_sig);
        } else if (staged_signature(ctx, g)) {
            const TileRange all{0u, 0u, nullptr, nullptr, 0ull};
            if (first == kPassRank8)
                k_signature_staged<uint8_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st,
                                                                           reinterpret_cast<const uint8_t*>(g->d_rank), g->d_sig,
                                                                           all, 0);
            else if (first == kPassRank16)
                k_signature_staged<uint16_t><<<blocks, kTileThreads, 0, s>>>(
                    g->d_as, g->d_st, reinterpret_cast<const uint16_t*>(g->d_rank), g->d_sig, all, 0);
            else
                k_signature_staged<uint32_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->d_sig, all, 0);
        } else if (first == kPassRank8 && g->hot_active && (ctx->opts.sig_kernel == 4 || (ctx->opts.sig_kernel == 0 && g->hot_tma))) {
            // the default when the tensor map could be made; asked for
            // explicitly, its absence is an error
            if (!g->hot_tma)
                return rbsc_fail(ctx, RBSC_ERR_CUDA, "sig_kernel 4: no tensor map for the hot heads (%d)", g->hot_tma_err);
            const uint8_t* cr = reinterpret_cast<const uint8_t*>(g->d_rank);
            const unsigned hgrid = std::min<unsigned>((unsigned)ctx->sm_count, ceil_div<uint32_t>(g->ntiles, kHotThreads / 32));
            const size_t smem = hot_tma_smem(g->hot_bytes);
            if (g->weighted)
                k_signature_hot_tma<true><<<hgrid, kHotThreads, smem, s>>>(g->hot_tmap, g->d_as, g->d_st, cr, g->d_hot_rank,
                                                                           g->hot_bytes, g->d_sig);
            else
                k_signature_hot_tma<false><<<hgrid, kHotThreads, smem, s>>>(g->hot_tmap, g->d_as, g->d_st, cr, g->d_hot_rank,
                                                                            g->hot_bytes, g->d_sig);
        } else if (first == kPassRank8 && g->hot_active) {
            const uint8_t* cr = reinterpret_cast<const uint8_t*>(g->d_rank);
            const unsigned hgrid = std::min<unsigned>((unsigned)ctx->sm_count, ceil_div<uint32_t>(g->ntiles, kHotThreads / 32));
            if (g->weighted)
                k_signature_hot<true><<<hgrid, kHotThreads, g->hot_bytes, s>>>(g->d_as, g->d_st, cr, g->d_hot_idx, g->d_hot_rank,
                                                                              g->hot_bytes, g->d_sig);
            else
                k_signature_hot<false><<<hgrid, kHotThreads, g->hot_bytes, s>>>(g->d_as, g->d_st, cr, g->d_hot_idx,
                                                                               g->d_hot_rank, g->hot_bytes, g->d_sig);
        } else if (first == kPassRank8) {
            const uint8_t* cr = reinterpret_cast<const uint8_t*>(g->d_rank);
            if (g->weighted)
                k_signature<true, uint8_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, cr, g->d_sig);
            else
                k_signature<false, uint8_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, cr, g->d_sig);
        } else if (first == kPassRank16) {
            const uint16_t* cr = reinterpret_cast<const uint16_t*>(g->d_rank);
            if (g->weighted)
                k_signature<true, uint16_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, cr, g->d_sig);
            else
                k_signature<false, uint16_t><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, cr, g->d_sig);
        } else if (g->weighted) {
            k_signature_auto<true><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->d_sig);
        } else {
            k_signature_auto<false><<<blocks, kTileThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->d_sig);
        }
    }
    if (t) CK(cudaEventRecord(t->ev[2], s));
    if (first != kPassFull) CK(cudaEventRecord(ctx->ev_sig[1], s));
    if (!hash) {
        CKS(launch_sort_relabel(ctx, g, s));
        if (t) CK(cudaEventRecord(t->ev[3], s));
    } else {
        CK(cudaStreamWaitEvent(s, ctx->ev_join, 0));
        ++rbsc::launch_counter();
        k_insert_list<<<ngrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->d_sig, g->d_tab8, g->log2tab, g->d_slot,
                                                     g->d_joined);
        if (t) CK(cudaEventRecord(t->ev[3], s));
        ++rbsc::launch_counter();
        k_relabel_list<<<ngrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->d_tab8, g->d_slot, g->d_sig,
                                                      g->d_joined);
    }
    ++rbsc::launch_counter();
    k_follow<<<ngrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_pairs, g->d_col[0]);
    if (t) CK(cudaEventRecord(t->ev[4], s));
    ++rbsc::launch_counter();
    k_fixpoint<kFixHash><<<1, 1, 0, s>>>(g->d_st, g->d_as, hash ? 1 : 0);
    // compaction for the next pass
    ++rbsc::launch_counter();
    k_compact_nodes<<<ngrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->cb);
    if (g->compact_arcs) {
        const unsigned kgrid = persistent_grid(ctx, g->K, kNodeThreads);
        const unsigned agrid = persistent_grid(ctx, ceil_div<uint64_t>(g->m, 16), kNodeThreads);
        ++rbsc::launch_counter();
        k_compact_rows<<<kgrid, kNodeThreads, 0, s>>>(g->d_as, g->d_st, g->d_col[0], g->cb);
        ++rbsc::launch_counter();
        k_compact_decide<<<1, 1, 0, s>>>(g->d_as, g->d_st, g->cb);
        if (g->arcs_on_host) {
            // source arcs in host memory: a coalesced copy, then the bookkeeping
            ++rbsc::launch_counter();
            k_compact_copy_tiles<<<persistent_grid(ctx, g->ntiles, kNodeThreads / 32), kNodeThreads, 0, s>>>(g->d_as, g->cb);
            ++rbsc::launch_counter();
            k_compact_arcs<false><<<agrid, kNodeThreads, 0, s>>>(g->d_as, g->cb, g->d_sig);
        } else {
            ++rbsc::launch_counter();
            k_compact_arcs<true><<<agrid, kNodeThreads, 0, s>>>(g->d_as, g->cb, g->d_sig);
        }
    }
    ++rbsc::launch_counter();
    // no hand-off to the persistent kernel from a pass over host arcs: the
    // next pass sees whether the compaction brought them into device memory
    const bool persist = hash && !ctx->opts.no_persist && !g->arcs_on_host;
    const uint64_t plim = persist_limit(ctx);
    k_compact_finalize<<<1, 1, 0, s>>>(g->d_as, g->d_st, g->cb, persist ? plim : 0ull, (uint32_t)std::min<uint64_t>(plim, 0xffffffffull),
                                       h, use_handle);
    if (t) CK(cudaEventRecord(t->ev[5], s));
    CK(cudaGetLastError());
    return RBSC_OK;
}

static rbsc_status build_loop_graph(rbsc_ctx* ctx, rbsc_graph* g)
{
    if (g->loop_exec && g->loop_relabel == ctx->opts.relabel && g->loop_no_persist == ctx->opts.no_persist &&
        g->loop_persist_log2 == ctx->opts.persist_log2 && g->loop_grid_per_sm == ctx->opts.grid_per_sm)
        return RBSC_OK;
    if (g->loop_exec) cudaGraphExecDestroy(g->loop_exec);
    if (g->loop_graph) cudaGraphDestroy(g->loop_graph);
    g->loop_exec = nullptr;
    g->loop_graph = nullptr;
    CKS(ensure_sort_relabel_bufs(ctx, g));
    CK(cudaGraphCreate(&g->loop_graph, 0));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g->loop_graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g->loop_graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return rbsc_cuda_fail(ctx, e, "cudaStreamBeginCaptureToGraph", __LINE__);
    }
    const uint64_t lc0 = rbsc::launch_counter();
    rbsc_status st = launch_pass(ctx, g, cs, h, 1);
    g->body_kernels = rbsc::launch_counter() - lc0;
    rbsc::launch_counter() = lc0;  // captured, not launched
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    if (st != RBSC_OK) return st;
    if (e != cudaSuccess) return rbsc_cuda_fail(ctx, e, "cudaStreamEndCapture", __LINE__);
    CK(cudaGraphInstantiate(&g->loop_exec, g->loop_graph, 0));
    g->loop_relabel = ctx->opts.relabel;
    g->loop_no_persist = ctx->opts.no_persist;
    g->loop_persist_log2 = ctx->opts.persist_log2;
    g->loop_grid_per_sm = ctx->opts.grid_per_sm;
    return RBSC_OK;
}

static rbsc_status read_state(rbsc_ctx* ctx, rbsc_graph* g)
{
    CK(cudaMemcpyAsync(g->h_st, g->d_st, sizeof(RoundState), cudaMemcpyDeviceToHost, ctx->stream));
    // a streamed graph: did the last pass's compaction bring the arcs into
    // device memory?
    const uint32_t* idx = nullptr;
    if (g->arcs_on_host)
        CK(cudaMemcpyAsync(&idx, &g->d_as->idx, sizeof idx, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (g->arcs_on_host) g->arcs_on_host = idx == g->d_idx;
    return RBSC_OK;
}

static rbsc_status run_passes(rbsc_ctx* ctx, rbsc_graph* g, rbsc_kernel_times* kt, uint64_t* graph_kernels);
static rbsc_status run_persistent(rbsc_ctx* ctx, rbsc_graph* g, rbsc_kernel_times* kt);

static rbsc_status run_loop(rbsc_ctx* ctx, rbsc_graph* g, rbsc_kernel_times* kt, uint64_t* graph_kernels,
                            int first = kPassFull, uint32_t c0 = 0)
{
    bool handoff = false;
    if (first != kPassFull) {
        // the first pass with its narrow gather, launched from the host; the
        // remaining passes below
        PassTimer t;
        if (kt)
            for (auto& e : t.ev) CK(cudaEventCreate(&e));
        ActiveSet before;
        if (kt) {
            CK(cudaMemcpyAsync(&before, g->d_as, sizeof before, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        CKS(ensure_sort_relabel_bufs(ctx, g));
        rbsc_status st = launch_pass(ctx, g, ctx->stream, cudaGraphConditionalHandle(), 0, kt ? &t : nullptr, first, c0);
        if (st == RBSC_OK) st = read_state(ctx, g);
        if (st == RBSC_OK) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev_sig[0], ctx->ev_sig[1]);
            g->first_sig_ms = ms;
            g->first_sig_arcs = first == kPassUniform ? 0 : g->m;
        }
        if (st == RBSC_OK && kt) {
            float ms[5];
            for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], t.ev[i], t.ev[i + 1]);
            float* pm = kt->pass_ms[0];
            pm[0] = ms[1];
            pm[1] = ms[2];
            pm[2] = ms[3];
            pm[3] = ms[0] + ms[4];
            kt->pass_arcs[0] = first == kPassUniform ? 0 : before.m;
            kt->pass_nodes[0] = before.nnodes;
            kt->passes = 1;
            kt->other_ms += ms[0] + ms[4];
            kt->signature_ms += ms[1];
            kt->insert_ms += ms[2];
            kt->relabel_ms += ms[3];
        }
        if (kt)
            for (auto& e : t.ev) cudaEventDestroy(e);
        if (st != RBSC_OK) return st;
        if (g->h_st->done || g->h_st->error) return RBSC_OK;
        handoff = g->h_st->handoff != 0;
    }
    if (!handoff) {
        CKS(run_passes(ctx, g, kt, graph_kernels));
        handoff = g->h_st->handoff != 0;
    }
    if (handoff && !g->h_st->done && !g->h_st->error) CKS(run_persistent(ctx, g, kt));
    return RBSC_OK;
}

// The small-set tail of the refinement: one cooperative launch of
// k_refine_persistent (all blocks resident, bounded grid barriers).
static rbsc_status run_persistent(rbsc_ctx* ctx, rbsc_graph* g, rbsc_kernel_times* kt)
{
    cudaStream_t s = ctx->stream;
    // signature phase: one row per lane when the active rows are short (mean
    // at most 4 arcs), else the tile fold (rows of a web graph's tail)
    const RoundState& hs = *g->h_st;
    const bool rows = ctx->opts.persist_sig == 1 ||
                      (ctx->opts.persist_sig != 2 && (uint64_t)hs.active_arcs <= 4ull * std::max<uint32_t>(hs.active_rows, 1u));
    const void* kern = rows ? (const void*)k_refine_persistent<true> : (const void*)k_refine_persistent<false>;
    int bps = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kNodeThreads, 0));
    bps = std::max(1, bps);
    // as many blocks as fit (measured best on R-MAT-24 and cnr-2000: the
    // phases are latency-bound, and fewer blocks do not make the barriers
    // cheap enough to pay for it), unless the options fix the count
    const int want = ctx->opts.persist_bps > 0 ? ctx->opts.persist_bps : bps;
    const unsigned grid = (unsigned)std::min(bps, want) * (unsigned)ctx->sm_count;
    CK(cudaMemsetAsync(g->d_gsync, 0, sizeof(GridSync), s));
    // the persistent kernel's per-parity counters and representative flags
    CK(cudaMemsetAsync(g->d_st->pcount, 0, sizeof g->d_st->pcount + sizeof g->d_st->prep, s));
    PersistArgs a;
    a.as = g->d_as;
    a.st = g->d_st;
    a.col = g->d_col[0];
    a.sig = g->d_sig;
    a.tab = g->d_tab;
    a.tab8 = g->d_tab8;
    // windows of at most 2^20 entries (8 MB to zero per pass): the 8-byte table
    a.use8 = g->h_st->active_nodes <= (1u << 19) ? 1 : 0;
    a.log2tab = g->log2tab;
    a.tab_entries = 1ull << g->log2tab;
    a.slot = g->d_slot;
    a.pairs = g->d_pairs;
    a.joined = g->d_joined;
    a.gs = g->d_gsync;
    a.weighted = g->weighted ? 1 : 0;
    void* args[] = {&a};
    const uint32_t r0 = g->h_st->round;
    if (kt) CK(cudaEventRecord(ctx->ev[2], s));
    ++rbsc::launch_counter();
    CK(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kNodeThreads), args, 0, s));
    if (kt) CK(cudaEventRecord(ctx->ev[3], s));
    CKS(read_state(ctx, g));
    if (kt) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        kt->persist_ms += ms;
        kt->persist_passes += g->h_st->round - r0;
    }
    if (g->h_st->error & kErrBarrier) return rbsc_fail(ctx, RBSC_ERR_DEVICE, "persistent kernel: a grid barrier timed out");
    return RBSC_OK;
}

// Passes with the active set still large: the CUDA-graph loop (or the
// host-driven loop), until the fixpoint, an error or the hand-off.
static rbsc_status run_passes(rbsc_ctx* ctx, rbsc_graph* g, rbsc_kernel_times* kt, uint64_t* graph_kernels)
{
    // passes over host arcs run from the host (each streams its chunks)
    // until a compaction brings the active arcs into device memory
    const bool graph_loop = ctx->opts.use_graph && !kt && !g->oneshot;
    if (graph_loop && g->arcs_on_host) {
        CKS(ensure_sort_relabel_bufs(ctx, g));
        while (g->arcs_on_host) {
            CKS(launch_pass(ctx, g, ctx->stream, cudaGraphConditionalHandle(), 0));
            CKS(read_state(ctx, g));
            if (g->h_st->done || g->h_st->error || g->h_st->handoff) return RBSC_OK;
        }
    }
    if (graph_loop) {
        CKS(build_loop_graph(ctx, g));
        const uint32_t r0 = g->h_st->round;
        CK(cudaGraphLaunch(g->loop_exec, ctx->stream));
        CKS(read_state(ctx, g));
        *graph_kernels += g->body_kernels * (uint64_t)(g->h_st->round - r0);
    } else {
        CKS(ensure_sort_relabel_bufs(ctx, g));
        PassTimer t;
        if (kt)
            for (auto& e : t.ev) CK(cudaEventCreate(&e));
        for (;;) {
            ActiveSet before;
            if (kt) {
                CK(cudaMemcpyAsync(&before, g->d_as, sizeof before, cudaMemcpyDeviceToHost, ctx->stream));
                CK(cudaStreamSynchronize(ctx->stream));
            }
            rbsc_status st = launch_pass(ctx, g, ctx->stream, cudaGraphConditionalHandle(), 0, kt ? &t : nullptr);
            if (st == RBSC_OK) st = read_state(ctx, g);
            if (st == RBSC_OK && kt) {
                float ms[5];
                for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], t.ev[i], t.ev[i + 1]);
                if (kt->passes < 32) {
                    float* pm = kt->pass_ms[kt->passes];
                    pm[0] = ms[1];
                    pm[1] = ms[2];
                    pm[2] = ms[3];
                    pm[3] = ms[0] + ms[4];
                    kt->pass_arcs[kt->passes] = before.m;
                    kt->pass_nodes[kt->passes] = before.nnodes;
                }
                kt->passes += 1;
                kt->other_ms += ms[0] + ms[4];
                kt->signature_ms += ms[1];
                kt->insert_ms += ms[2];
                kt->relabel_ms += ms[3];
            }
            if (st != RBSC_OK || g->h_st->done || g->h_st->error || g->h_st->handoff) {
                if (kt)
                    for (auto& e : t.ev) cudaEventDestroy(e);
                if (st != RBSC_OK) return st;
                break;
            }
        }
    }
    return RBSC_OK;
}

// Clears what the set-up of the active set expects to be clear: the words of
// the arc-less groups (k_group_reps) and the signatures of the rows that
// cross a tile edge (the first pass adds into them).
static rbsc_status clear_setup_words(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s)
{
    if (g->nsplit) {
        ++rbsc::launch_counter();
        k_zero_rows<<<grid_for(g->nsplit, 256), 256, 0, s>>>(g->d_split, g->nsplit, g->d_sig);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(g->d_grep, 0xff, 4 * (size_t)g->n, s));
    CK(cudaMemsetAsync(g->d_gcnt, 0, 4 * (size_t)g->n, s));
    return RBSC_OK;
}

// Resets the active set to the whole graph and builds the node list and the
// follower pairs from the current colouring (after the initial or a repair
// pass).  side_cleared: clear_setup_words ran on the side stream, which
// recorded ev_join after it.
static rbsc_status init_active_set(rbsc_ctx* ctx, rbsc_graph* g, bool side_cleared = false)
{
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n;
    ActiveSet a;
    std::memset(&a, 0, sizeof a);
    a.rows = g->d_rows;
    a.roff = g->d_roff;
    a.roff64 = g->off32 ? 0u : 1u;
    a.tile_row = g->d_tile_row;
    a.head8 = g->d_head8;
    a.idx = g->d_idx;
    a.wt = g->d_wt;
    a.split = g->d_split;
    a.m = g->m;
    a.K = g->K;
    a.ntiles = g->ntiles;
    a.nsplit = g->nsplit;
    a.nodes = g->cb.nodes[0];
    a.compact_arcs = g->compact_arcs ? 1u : 0u;
    a.dst_cap = g->host_arcs ? g->resident_cap : std::max<uint64_t>(ceil_div<uint64_t>(3 * g->m, 4), 1);
    a.arcctr = 0;
    g->arcs_on_host = g->host_arcs;
    *g->h_as = a;
    CK(cudaMemcpyAsync(g->d_as, g->h_as, sizeof a, cudaMemcpyHostToDevice, s));
    if (side_cleared) CK(cudaStreamWaitEvent(s, ctx->ev_join, 0));
    else CKS(clear_setup_words(ctx, g, s));
    const unsigned lgrid = (unsigned)std::min<uint64_t>((uint64_t)ctx->sm_count * 8, ceil_div<uint64_t>(n, 256));
    ++rbsc::launch_counter();
    k_group_reps<<<lgrid, 256, 0, s>>>(n, g->d_off, g->d_initlab, g->d_grep, g->d_gcnt);
    ++rbsc::launch_counter();
    k_build_lists<<<lgrid, kNodeThreads, 0, s>>>(n, g->d_off, g->d_initlab, g->d_col[0], g->d_grep, g->d_gcnt, g->d_as,
                                                 g->cb.nodes[0], g->d_pairs);
    ++rbsc::launch_counter();
    k_publish_list<<<1, 1, 0, s>>>(g->d_as);
    CK(cudaGetLastError());
    return RBSC_OK;
}

// Exact check of the current fixpoint.  Returns the number of failing nodes in
// *nfail (0 = the partition is the coarsest stable one).
static rbsc_status verify_fixpoint(rbsc_ctx* ctx, rbsc_graph* g, uint32_t* nfail, uint32_t* out)
{
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n;
    const uint32_t* col = g->d_col[0];
    if (!g->d_vflag) {
        CKS(dev_alloc(ctx, (void**)&g->d_vflag, 4 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_vrow, 4 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_vdeg, 8 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_fail, 4 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_vl8, 4 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_vl32, 4 * ((size_t)n + 1)));
        CKS(dev_alloc(ctx, (void**)&g->d_vllong, 4 * ((size_t)n + 1)));
        // zero between checks from here on: a check that sets flags clears
        // them after use (the long-row path below, the repair pass)
        CK(cudaMemsetAsync(g->d_vflag, 0, 4 * ((size_t)n + 1), ctx->stream));
        CK(cudaMemsetAsync(g->d_fail, 0, 4 * ((size_t)n + 1), ctx->stream));
    }
    uint32_t* counts = reinterpret_cast<uint32_t*>(g->d_small);          // [0..3] list sizes, failures
    uint64_t* tot = reinterpret_cast<uint64_t*>(g->d_small) + 4;          // [0] rows, [1] keys of the global path
    CK(cudaMemsetAsync(g->d_small, 0, 64, s));
    if (g->verify_dirty) {  // a check or repair that ended early left flags set
        CK(cudaMemsetAsync(g->d_vflag, 0, 4 * ((size_t)n + 1), s));
        CK(cudaMemsetAsync(g->d_fail, 0, 4 * ((size_t)n + 1), s));
    }
    g->verify_dirty = true;
    // the arc view: the graph's own arrays, or -- when those are in host
    // memory and the active set was compacted into device memory -- the
    // compacted rows (every row the check reads is among them)
    const uint64_t* vstart = g->d_off;
    const uint32_t* vidx = g->d_idx;
    const uint64_t* vwt = g->d_wt;
    if (g->host_arcs && !g->arcs_on_host) {
        if (!g->d_vstart) CKS(dev_alloc(ctx, (void**)&g->d_vstart, 8 * ((size_t)n + 1)));
        ActiveSet as;
        CK(cudaMemcpyAsync(&as, g->d_as, sizeof as, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        ++rbsc::launch_counter();
        k_verify_starts<<<persistent_grid(ctx, as.K, 256), 256, 0, s>>>(g->d_as, g->d_vstart);
        CK(cudaGetLastError());
        vstart = g->d_vstart;
        vidx = as.idx;
        vwt = as.wt;
    }
    VerifyLists vl{g->d_vl8, g->d_vl32, g->d_vllong, counts};
    ++rbsc::launch_counter();
    k_verify_classify<<<persistent_grid(ctx, n, 256), 256, 0, s>>>(n, col, g->d_initlab, g->d_off, g->weighted ? 1 : 0, vl,
                                                                  g->d_vflag, g->d_fail, out);
    const unsigned sgrid = persistent_grid(ctx, n, 256);
    ++rbsc::launch_counter();
    k_verify_short<8><<<sgrid, 256, 0, s>>>(n, g->d_vl8, counts + 0, col, g->d_off, vstart, vidx, g->d_fail, counts + 3);
    ++rbsc::launch_counter();
    k_verify_short<32><<<sgrid, 256, 0, s>>>(n, g->d_vl32, counts + 1, col, g->d_off, vstart, vidx, g->d_fail, counts + 3);
    CK(cudaGetLastError());
    uint32_t hc[4];
    CK(cudaMemcpyAsync(hc, counts, sizeof hc, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hc[2] > 0) {
        // global path for long / weighted rows: sort each flagged row's colours
        CKS(ensure_temp(ctx, g, scan_temp_bytes<uint64_t>((uint64_t)n + 1) + 1024));
        ++rbsc::launch_counter();
        k_verify_mark<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_off, g->d_vflag, g->d_vdeg);
        CK(cudaGetLastError());
        CK((exclusive_scan<uint32_t, uint32_t>(g->d_vflag, g->d_vrow, n, (uint32_t*)tot, g->d_tmp, s)));
        CK((exclusive_scan<uint64_t, uint64_t>(g->d_vdeg, g->d_vdeg, n, tot + 1, g->d_tmp, s)));
        uint64_t ht[2];
        CK(cudaMemcpyAsync(ht, tot, sizeof ht, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const uint32_t nrows = (uint32_t)ht[0];
        const uint64_t nkeys = ht[1];
        if (nkeys >= (1ull << 32))
            return rbsc_fail(ctx, RBSC_ERR_TOO_LARGE, "exact check: %llu arcs in long rows (limit 2^32)", (unsigned long long)nkeys);
        if (nkeys > g->key_cap) {
            dev_free(g->ctx, (void*&)g->d_keys[0]);
            dev_free(g->ctx, (void*&)g->d_keys[1]);
            dev_free(g->ctx, (void*&)g->d_vals[0]);
            dev_free(g->ctx, (void*&)g->d_vals[1]);
            g->key_cap = 0;
            CKS(dev_alloc(ctx, (void**)&g->d_keys[0], 8 * nkeys));
            CKS(dev_alloc(ctx, (void**)&g->d_keys[1], 8 * nkeys));
            if (g->weighted) {
                CKS(dev_alloc(ctx, (void**)&g->d_vals[0], 8 * nkeys));
                CKS(dev_alloc(ctx, (void**)&g->d_vals[1], 8 * nkeys));
            }
            g->key_cap = nkeys;
        }
        const unsigned long long* keys = g->d_keys[0];
        const unsigned long long* vals = g->weighted ? g->d_vals[0] : nullptr;
        if (nkeys > 0) {
            ++rbsc::launch_counter();
            k_verify_keys<<<grid_for(n, 128), 128, 0, s>>>(n, col, g->d_off, vstart, vidx, vwt, g->d_vflag, g->d_vrow,
                                                          g->d_vdeg, g->d_keys[0], g->weighted ? g->d_vals[0] : nullptr);
            CK(cudaGetLastError());
            CKS(ensure_temp(ctx, g, radix_temp_bytes(nkeys)));
            const int bits = 31 + (int)log2_ceil(std::max<uint32_t>(nrows, 1));
            bool in_alt = false;
            CK(radix_sort<unsigned long long>(g->d_keys[0], g->d_keys[1], g->weighted ? g->d_vals[0] : (unsigned long long*)nullptr,
                                              g->weighted ? g->d_vals[1] : (unsigned long long*)nullptr, nkeys, 0, bits, g->d_tmp, s,
                                              &in_alt));
            if (in_alt) {
                keys = g->d_keys[1];
                vals = g->weighted ? g->d_vals[1] : nullptr;
            }
        }
        const unsigned cgrid = (unsigned)std::min<uint64_t>((uint64_t)ctx->sm_count * 16, grid_for((uint64_t)hc[2] * 32, 256));
        ++rbsc::launch_counter();
        k_verify_compare<<<cgrid, 256, 0, s>>>(g->d_vllong, counts + 2, col, g->d_initlab, g->d_off, g->d_vdeg, keys, vals,
                                               g->d_fail, counts + 3);
        CK(cudaGetLastError());
        CK(cudaMemsetAsync(g->d_vflag, 0, 4 * ((size_t)n + 1), s));
        CK(cudaMemcpyAsync(hc, counts, sizeof hc, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    *nfail = hc[3];
    g->verify_dirty = hc[3] != 0;  // failure flags stay set for the repair pass
    return RBSC_OK;
}

// Splits the nodes that failed the exact check away from their blocks, then
// restarts the active set from the whole graph.
static rbsc_status repair_pass(rbsc_ctx* ctx, rbsc_graph* g)
{
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n;
    const unsigned clear_grid = (unsigned)std::min<uint64_t>(ctx->sm_count * 8ull, grid_for(1ull << g->log2tab, 256));
    ++rbsc::launch_counter();
    k_clear_table<<<clear_grid, 256, 0, s>>>(g->d_st, g->d_tab, 1ull << g->log2tab);
    ++rbsc::launch_counter();
    k_insert_all<kModeRepair><<<persistent_grid(ctx, n, kNodeThreads), kNodeThreads, 0, s>>>(n, g->d_st, g->d_col[0], g->d_fail,
                                                                                             g->d_tab, g->log2tab, g->d_slot);
    CK(cudaMemsetAsync(g->d_fail, 0, 4 * ((size_t)n + 1), s));  // the failure flags are consumed
    g->verify_dirty = false;
    ++rbsc::launch_counter();
    k_relabel_all<<<persistent_grid(ctx, n, kNodeThreads), kNodeThreads, 0, s>>>(n, g->d_col[0], g->d_tab, g->d_slot, nullptr);
    ++rbsc::launch_counter();
    k_fixpoint<kFixRepair><<<1, 1, 0, s>>>(g->d_st, g->d_as, 0);
    CK(cudaGetLastError());
    // every row signature is recomputed from scratch on the whole graph
    CK(cudaMemsetAsync(g->d_sig, 0, sizeof(Sig) * (size_t)n, s));
    return init_active_set(ctx, g);
}

// The whole refinement of a resident graph, device pointers in and out.
rbsc_status refine_resident(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init, uint32_t* d_out, rbsc_stats* stats,
                            rbsc_kernel_times* kt)
{
    CK(cudaSetDevice(ctx->device));
    const uint64_t lc0 = rbsc::launch_counter();
    uint64_t graph_kernels = 0;
    cudaStream_t s = ctx->stream;
    const uint32_t n = g->n;
    if (stats) std::memset(stats, 0, sizeof *stats);
    if (n == 0) {
        if (stats) stats->done = stats->verified = 1;
        return RBSC_OK;
    }
    CKS(ensure_refine_bufs(ctx, g));
    g->first_sig_ms = 0.f;
    g->first_sig_arcs = 0;
    g->streamed_bytes = 0;
    g->streamed_passes = 0;
    // the joined flags, the arc-less groups' words and the split rows'
    // signatures are cleared on the side stream beside the initial pass
    // (k_insert_init is bound by issue, not by HBM); the set-up waits for them
    CK(cudaEventRecord(ctx->ev_fork, s));
    CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
    CK(cudaMemsetAsync(g->d_joined, 0, 4 * (size_t)n, ctx->side));
    CKS(clear_setup_words(ctx, g, ctx->side));
    CK(cudaEventRecord(ctx->ev_join, ctx->side));
    RoundState& hs = *g->h_st;
    std::memset(&hs, 0, sizeof hs);
    hs.max_rounds = ctx->opts.max_rounds ? ctx->opts.max_rounds : (n + 1u);
    hs.seed = ctx->opts.seed;
    hs.hash_bits = ctx->opts.test_hash_bits < 0 ? 64u : (uint32_t)ctx->opts.test_hash_bits;
    hs.stamp = g->next_stamp;
    hs.clear_pending = 0;
    CK(cudaEventRecord(ctx->ev[0], s));
    if (d_init) {
        CK(cudaMemcpyAsync(g->d_st, &hs, sizeof hs, cudaMemcpyHostToDevice, s));
        const unsigned igrid = (unsigned)std::min<uint64_t>((uint64_t)ctx->sm_count * 8, ceil_div<uint64_t>(n, kNodeThreads));
        const uint32_t chunk = (uint32_t)(ceil_div<uint64_t>(ceil_div<uint64_t>(n, igrid), kNodeThreads) * kNodeThreads);
        ++rbsc::launch_counter();
        k_insert_init<<<igrid, kNodeThreads, 0, s>>>(n, chunk, g->d_st, d_init, g->d_tab, g->log2tab, g->d_slot, g->d_srank);
        ++rbsc::launch_counter();
        k_relabel_all<<<persistent_grid(ctx, n, kNodeThreads), kNodeThreads, 0, s>>>(n, g->d_col[0], g->d_tab, g->d_slot,
                                                                                        g->d_initlab, g->d_st, g->d_srank,
                                                                                        g->d_rank);
        ++rbsc::launch_counter();
        k_fixpoint<kFixInit><<<1, 1, 0, s>>>(g->d_st, g->d_as, 0);
        CK(cudaGetLastError());
    } else {
        hs.prev = 1;
        hs.round_blocks[0] = 1;
        CK(cudaMemcpyAsync(g->d_st, &hs, sizeof hs, cudaMemcpyHostToDevice, s));
        ++rbsc::launch_counter();
        k_fill_uniform<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0]);
        ++rbsc::launch_counter();
        k_strip_labels<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0], g->d_initlab);
        CK(cudaGetLastError());
    }
    // The state after the initial pass (its block count picks the first
    // pass's gather width) comes back while the setup kernels run: the host
    // waits for that copy (ev[7]), not for the setup.  The profile path keeps
    // a synchronisation between the phases to time each.
    if (kt) {
        CKS(read_state(ctx, g));
        CK(cudaEventRecord(ctx->ev[4], s));
        CK(cudaEventSynchronize(ctx->ev[4]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[4]);
        kt->init_ms = ms;
    } else {
        CK(cudaMemcpyAsync(g->h_st, g->d_st, sizeof(RoundState), cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(ctx->ev[7], s));
    }
    CKS(init_active_set(ctx, g, true));
    if (kt) {
        CK(cudaEventRecord(ctx->ev[5], s));
        CK(cudaEventSynchronize(ctx->ev[5]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
        kt->setup_ms = ms;
    }
    CK(cudaEventRecord(ctx->ev[6], s));  // end of init + setup, read after the refinement
    if (!kt) CK(cudaEventSynchronize(ctx->ev[7]));
    const uint32_t initial_blocks = hs.prev;

    // first pass: few initial classes -> gather their dense ranks (1 or 2
    // bytes per node); one class -> no gather at all
    int first = kPassFull;
    uint32_t c0 = 0;
    if (g->m > 0 && ctx->opts.relabel != RBSC_RELABEL_SORT) {
        if (initial_blocks == 1) {
            first = kPassUniform;
            c0 = 0;  // the one class is labelled by node 0
        } else if (initial_blocks <= 65536) {
            first = initial_blocks <= 256 ? kPassRank8 : kPassRank16;
        }
        // k_relabel_all wrote the ranks when k_insert_init ranked every class;
        // otherwise: ranks of the class heads in label order, by a scan
        if ((first == kPassRank8 || first == kPassRank16) && !(d_init && !hs.rank_bad && hs.ranks == initial_blocks)) {
            CKS(ensure_temp(ctx, g, scan_temp_bytes<uint32_t>((uint64_t)n + 1) + 1024));
            ++rbsc::launch_counter();
            k_class_heads<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0], g->d_slot);
            CK((exclusive_scan<uint32_t, uint32_t>(g->d_slot, g->d_slot, n, (uint32_t*)nullptr, g->d_tmp, s)));
            ++rbsc::launch_counter();
            if (first == kPassRank8)
                k_class_ranks<uint8_t><<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0], g->d_slot, (uint8_t*)g->d_rank);
            else
                k_class_ranks<uint16_t><<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0], g->d_slot, (uint16_t*)g->d_rank);
            CK(cudaGetLastError());
        }
    }
    // hot heads: the first pass reads the ranks of the most pointed-to nodes
    // from shared memory
    g->hot_active = false;
    if (first == kPassRank8 && hot_wanted(ctx, g)) {
        bool ready = false;
        CKS(build_hot(ctx, g, &ready));
        if (ready) {
            ++rbsc::launch_counter();
            k_hot_ranks<<<grid_for(g->hot_bytes, 256), 256, 0, s>>>(g->hot_n, g->hot_bytes, g->d_hot_node,
                                                                   reinterpret_cast<const uint8_t*>(g->d_rank), g->d_hot_rank);
            CK(cudaGetLastError());
            g->hot_active = true;
        }
    }

    float verify_ms = 0.f, loop_ms = 0.f;
    uint32_t repairs = 0;
    uint32_t* out = d_out ? d_out : g->d_out;
    bool labels_out = false;  // a passed exact check wrote them
    for (;;) {
        if (hs.error) break;
        CK(cudaEventRecord(ctx->ev[4], s));
        CKS(run_loop(ctx, g, kt, &graph_kernels, first, c0));
        first = kPassFull;
        CK(cudaEventRecord(ctx->ev[5], s));
        CK(cudaEventSynchronize(ctx->ev[5]));
        {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
            loop_ms += ms;
        }
        if (hs.error) break;
        if (!ctx->opts.verify) break;
        CK(cudaEventRecord(ctx->ev[2], s));
        uint32_t nfail = 0;
        CKS(verify_fixpoint(ctx, g, &nfail, out));
        labels_out = nfail == 0;
        CK(cudaEventRecord(ctx->ev[3], s));
        CK(cudaEventSynchronize(ctx->ev[3]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        verify_ms += ms;
        if (nfail == 0) break;
        ++repairs;
        CKS(repair_pass(ctx, g));
        CKS(read_state(ctx, g));
    }
    g->next_stamp = hs.stamp;
    if (hs.error & kErrProbe) return rbsc_fail(ctx, RBSC_ERR_DEVICE, "relabel table overflow");
    if (hs.error & kErrStage) return rbsc_fail(ctx, RBSC_ERR_DEVICE, "signature: a staged tile copy did not complete");
    if (hs.error & kErrInput) return rbsc_fail(ctx, RBSC_ERR_INVALID, "an arc head is >= N");
    if (hs.error & kErrRounds) return rbsc_fail(ctx, RBSC_ERR_NOT_CONVERGED, "no fixpoint after %u passes", hs.round);
    if (!labels_out) {
        ++rbsc::launch_counter();
        k_strip_labels<<<grid_for(n, 256), 256, 0, s>>>(n, g->d_col[0], out);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ctx->ev[1], s));
    CK(cudaEventSynchronize(ctx->ev[1]));
    float total_ms = 0.f, init_ms = 0.f;
    cudaEventElapsedTime(&total_ms, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&init_ms, ctx->ev[0], ctx->ev[6]);
    if (stats) {
        stats->rounds = hs.round;
        stats->blocks = hs.prev;
        stats->done = 1;
        stats->verified = ctx->opts.verify ? 1u : 0u;
        stats->repairs = repairs;
        stats->initial_blocks = initial_blocks;
        stats->device_ms = total_ms;
        stats->verify_ms = verify_ms;
        for (int i = 0; i < 64 && i < kRoundLog; ++i) stats->round_blocks[i] = hs.round_blocks[i];
        stats->kernel_launches = rbsc::launch_counter() - lc0 + graph_kernels;
        stats->init_ms = init_ms;
        stats->loop_ms = loop_ms;
        stats->first_signature_ms = g->first_sig_ms;
        stats->first_signature_arcs = g->first_sig_arcs;
        stats->streamed_bytes = g->streamed_bytes;
        stats->streamed_passes = g->streamed_passes;
        stats->first_signature_hot = g->hot_active ? g->hot_n : 0u;
    }
    if (kt) kt->total_ms = total_ms;
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_graph_profile(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init_colors,
                                          rbsc_kernel_times* times, rbsc_stats* stats)
{
    if (!ctx || !g || !times) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    std::memset(times, 0, sizeof *times);
    return refine_resident(ctx, g, d_init_colors, nullptr, stats, times);
}

extern "C" rbsc_status rbsc_graph_refine_device(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init_colors,
                                                uint32_t* d_out_labels, rbsc_stats* stats)
{
    if (!ctx || !g) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    auto t0 = std::chrono::steady_clock::now();
    rbsc_status st = refine_resident(ctx, g, d_init_colors, d_out_labels, stats, nullptr);
    if (st == RBSC_OK && stats)
        stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

extern "C" rbsc_status rbsc_graph_refine(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* init_colors, uint32_t* out_labels,
                                         rbsc_stats* stats)
{
    if (!ctx || !g) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(ctx->device));
    auto t0 = std::chrono::steady_clock::now();
    CKS(ensure_refine_bufs(ctx, g));
    double h2d = 0, d2h = 0;
    const uint32_t* d_init = nullptr;
    if (init_colors && g->n && init_colors == g->h_init_loaded) {
        d_init = g->d_init;  // copied with the graph (one-shot call)
        g->h_init_loaded = nullptr;
    } else if (init_colors && g->n) {
        if (!g->d_init) CKS(dev_alloc(ctx, (void**)&g->d_init, 4 * (size_t)g->n));
        auto a = std::chrono::steady_clock::now();
        CK(cudaMemcpyAsync(g->d_init, init_colors, 4 * (size_t)g->n, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        h2d = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
        d_init = g->d_init;
    }
    CKS(refine_resident(ctx, g, d_init, nullptr, stats, nullptr));
    if (out_labels && g->n) {
        auto a = std::chrono::steady_clock::now();
        CK(cudaMemcpyAsync(out_labels, g->d_out, 4 * (size_t)g->n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        d2h = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    }
    if (stats) {
        stats->h2d_ms = h2d;
        stats->d2h_ms = d2h;
        stats->h2d_bytes = init_colors ? 4ull * g->n : 0;
        stats->d2h_bytes = out_labels ? 4ull * g->n : 0;
        stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_refine(rbsc_ctx* ctx, const rbsc_csr* host_graph, const uint32_t* init_colors,
                                   uint32_t* out_labels, rbsc_stats* stats)
{
    if (!ctx) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null context");
    auto t0 = std::chrono::steady_clock::now();
    rbsc_graph* g = nullptr;
    double up_ms = 0;
    uint64_t up_bytes = 0;
    // large unweighted graphs: the heads' copy overlaps the refinement
    const bool defer = host_graph && !host_graph->weights && host_graph->m >= (1ull << 22);
    CKS(graph_load(ctx, host_graph, false, &g, &up_ms, &up_bytes, defer, init_colors));
    g->oneshot = true;
    rbsc_status st = rbsc_graph_refine(ctx, g, init_colors, out_labels, stats);
    rbsc_graph_free(g);
    if (st == RBSC_OK && stats) {
        stats->h2d_ms += up_ms;
        stats->h2d_bytes += up_bytes;
        stats->time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

extern "C" rbsc_status rbsc_graph_degree_colors(rbsc_ctx* ctx, rbsc_graph* g, uint32_t* d_colors)
{
    if (!ctx || !g || !d_colors) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (g->n) {
        ++rbsc::launch_counter();
        k_degree_colors<<<grid_for(g->n, 256), 256, 0, ctx->stream>>>(g->n, g->d_off, d_colors);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return RBSC_OK;
}

// ---------------------------------------------------------------------------
// autotuning
// ---------------------------------------------------------------------------
extern "C" void rbsc_tune_space_default(rbsc_tune_space* sp)
{
    std::memset(sp, 0, sizeof *sp);
    const int32_t pl[] = {18, 20, 22, 24, -1};
    for (int32_t v : pl) sp->persist_log2[sp->n_persist++] = v;
    const int32_t gr[] = {4, 8, 16, 32};
    for (int32_t v : gr) sp->grid_per_sm[sp->n_grid++] = v;
    sp->relabel[sp->n_relabel++] = RBSC_RELABEL_HASH;
    sp->use_graph[sp->n_use_graph++] = 1;
    sp->use_graph[sp->n_use_graph++] = 0;
    sp->sig_kernel[sp->n_sig_kernel++] = 1;
    sp->sig_kernel[sp->n_sig_kernel++] = 2;
    sp->sig_kernel[sp->n_sig_kernel++] = 3;
    sp->sig_kernel[sp->n_sig_kernel++] = 4;
    sp->reps = 3;
}

extern "C" rbsc_status rbsc_graph_autotune(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init, const rbsc_tune_space* space,
                                           rbsc_opts* best, rbsc_tune_report* report)
{
    if (!ctx || !g || !best) return rbsc_fail(ctx, RBSC_ERR_INVALID, "null argument");
    rbsc_tune_space sp;
    if (space) sp = *space;
    else rbsc_tune_space_default(&sp);
    const rbsc_opts base = ctx->opts;
    auto list = [](const int32_t* v, uint32_t n, int32_t cur) {
        std::vector<int32_t> out(v, v + std::min<uint32_t>(n, RBSC_TUNE_MAX));
        if (out.empty()) out.push_back(cur);
        return out;
    };
    const auto pl = list(sp.persist_log2, sp.n_persist, base.persist_log2);
    const auto gr = list(sp.grid_per_sm, sp.n_grid, base.grid_per_sm);
    const auto rl = list(sp.relabel, sp.n_relabel, base.relabel);
    const auto ug = list(sp.use_graph, sp.n_use_graph, base.use_graph);
    const auto sks = list(sp.sig_kernel, sp.n_sig_kernel, base.sig_kernel);
    const uint32_t reps = sp.reps ? sp.reps : 3;
    rbsc_tune_report rep;
    std::memset(&rep, 0, sizeof rep);
    // one candidate: a warm-up refinement, then `reps` timed ones
    auto time_opts = [&](const rbsc_opts& o, double* med, uint32_t* blocks, uint32_t* rounds) -> rbsc_status {
        ctx->opts = o;
        rbsc_stats st;
        rbsc_status s = refine_resident(ctx, g, d_init, nullptr, &st, nullptr);
        if (s != RBSC_OK) return s;
        std::vector<double> t;
        for (uint32_t r = 0; r < reps; ++r) {
            s = refine_resident(ctx, g, d_init, nullptr, &st, nullptr);
            if (s != RBSC_OK) return s;
            t.push_back(st.device_ms);
        }
        std::sort(t.begin(), t.end());
        *med = t[t.size() / 2];
        *blocks = st.blocks;
        *rounds = st.rounds;
        return RBSC_OK;
    };
    uint32_t b0 = 0, r0 = 0;
    rbsc_status s = time_opts(base, &rep.default_ms, &b0, &r0);
    if (s != RBSC_OK) {
        ctx->opts = base;
        return s;
    }
    rbsc_opts chosen = base;
    double best_ms = rep.default_ms;
    for (int32_t p : pl)
        for (int32_t gsm : gr)
            for (int32_t r : rl)
                for (int32_t u : ug)
                  for (int32_t sk : sks) {
                    rbsc_opts o = base;
                    o.sig_kernel = sk;
                    o.persist_log2 = p;
                    o.no_persist = p < 0 ? 1 : base.no_persist;
                    o.grid_per_sm = gsm;
                    o.relabel = r;
                    o.use_graph = u;
                    double ms = 0;
                    uint32_t b = 0, rd = 0;
                    s = time_opts(o, &ms, &b, &rd);
                    if (s != RBSC_OK) {
                        ctx->opts = base;
                        return s;
                    }
                    const uint32_t i = rep.candidates++;
                    if (i < 64) {
                        rep.ms[i] = ms;
                        rep.opts[i] = o;
                    }
                    if (b != b0 || rd != r0) {
                        ++rep.failed;
                        continue;
                    }
                    if (ms < best_ms) {
                        best_ms = ms;
                        chosen = o;
                    }
                }
    ctx->opts = base;
    rep.best_ms = best_ms;
    *best = chosen;
    if (report) *report = rep;
    return RBSC_OK;
}
