// internal.h -- definitions shared by the host translation units of librbsc.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/rbsc.h"

#include "refine_kernels.cuh"

// Cached device (or pinned host) blocks of a context.  Buffers of freed
// graphs and temporaries go back here and are handed out again to later
// requests of about the same size: repeated one-shot refinements reuse
// memory instead of paying for cudaMalloc / cudaFree (and the first touch of
// fresh pages) every call.
struct MemPool {
    bool pinned = false;
    std::multimap<size_t, void*> free_blocks;  // size -> block, not in use
    std::unordered_map<void*, size_t> sizes;   // every block the pool allocated
    size_t cached = 0;                         // bytes in free_blocks
    size_t cap = (size_t)48 << 30;             // most bytes of unused blocks kept
};

struct rbsc_ctx {
    int device = 0;
    MemPool dpool;
    MemPool hpool{true};
    rbsc_opts opts{};
    cudaStream_t stream = nullptr;
    // [0]..[5] timing marks of a refinement; [6] the end of its initial pass
    // and setup kernels; [7] the copy of the state after the initial pass
    cudaEvent_t ev[8] = {};
    cudaEvent_t ev_sig[2] = {};  // around the host-launched first signature kernel
    // a pass clears the list table's window on this stream beside its
    // signature kernel (fork / join events, no timing)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int sm_count = 148;
    std::string err;
};

struct rbsc_graph {
    rbsc_ctx* ctx = nullptr;
    uint32_t n = 0;
    uint64_t m = 0;
    bool weighted = false;
    bool off32 = false;         // roff stored as uint32 (M < 2^32)
    uint64_t* d_off = nullptr;  // n+1 per-node arc offsets
    uint32_t* d_idx = nullptr;  // arc heads, padded to whole tiles
    uint64_t* d_wt = nullptr;   // weights (padded) or null
    uint32_t K = 0;             // non-empty rows
    uint32_t* d_rows = nullptr;
    void* d_roff = nullptr;
    uint32_t ntiles = 0;
    uint32_t* d_tile_row = nullptr;
    uint32_t nsplit = 0;
    uint32_t* d_split = nullptr;
    uint8_t* d_head8 = nullptr;  // row-head bitmap, one bit per arc

    // refinement state (allocated on first refine, reused)
    bool bufs = false;
    uint32_t* d_col[1] = {nullptr};  // colours, updated in place
    uint32_t* d_initlab = nullptr;
    rbsc::Sig* d_sig = nullptr;  // per-node signature (16 B)
    uint32_t* d_slot = nullptr;
    uint32_t* d_joined = nullptr;    // per node: pass in which a member joined its representative's class
    uint32_t* d_out = nullptr;
    void* d_rank = nullptr;          // first pass: dense class ranks (uint8 / uint16)
    // hot heads of the first pass (hot_kernels.cuh), built once per graph
    uint32_t* d_hot_idx = nullptr;   // heads, hot ones as kHotFlag | slot
    uint32_t* d_hot_node = nullptr;  // node of each hot slot
    uint8_t* d_hot_rank = nullptr;   // per refinement: class rank of each hot slot
    uint32_t hot_n = 0;              // hot slots
    uint32_t hot_bytes = 0;          // staged table: hot_n rounded up to 16
    int hot_state = 0;               // 0 not built, 1 built, -1 not applicable (no skew, no memory)
    CUtensorMap hot_tmap{};          // d_hot_idx as rows of 128 B, 16-row boxes, 128-byte swizzle
    bool hot_tma = false;            // hot_tmap encoded (k_signature_hot_tma can run)
    int hot_tma_err = 0;             // why not: -1 no driver entry point, -2 too many rows, else the CUresult
    uint32_t hot_log2 = 0;           // the size limit it was built (or rejected) for
    bool hot_active = false;         // the running refinement's first pass uses it
    uint32_t* d_srank = nullptr;     // rank of the initial class claimed at each table slot
    uint32_t* d_init = nullptr;
    rbsc::Entry* d_tab = nullptr;            // 16-byte entries: initial and repair passes
    unsigned long long* d_tab8 = nullptr;    // 8-byte entries: the list passes (same entry count)
    uint32_t log2tab = 0;
    uint32_t next_stamp = 1;
    rbsc::RoundState* d_st = nullptr;
    rbsc::RoundState* h_st = nullptr;  // pinned mirror
    void* d_small = nullptr;           // 256 B of counters
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;

    // active set (what the passes still work on)
    rbsc::ActiveSet* d_as = nullptr;
    rbsc::GridSync* d_gsync = nullptr;
    rbsc::ActiveSet* h_as = nullptr;  // pinned staging of the initial active set
    uint2* d_pairs = nullptr;        // (follower, representative)
    uint32_t* d_grep = nullptr;      // per initial label: smallest arc-less node
    uint32_t* d_gcnt = nullptr;      // per initial label: arc-less nodes
    rbsc::CompactBufs cb{};
    bool compact_arcs = false;

    // exact check
    uint32_t* d_vflag = nullptr;
    uint32_t* d_vrow = nullptr;
    uint32_t* d_vl8 = nullptr;
    uint32_t* d_vl32 = nullptr;
    uint32_t* d_vllong = nullptr;
    uint64_t* d_vdeg = nullptr;
    uint64_t* d_vstart = nullptr;    // exact check: row starts in the compacted active set
    uint32_t* d_fail = nullptr;
    bool verify_dirty = false;  // d_vflag / d_fail may hold flags (they are zero between checks otherwise)
    unsigned long long* d_keys[2] = {nullptr, nullptr};
    unsigned long long* d_vals[2] = {nullptr, nullptr};
    uint64_t key_cap = 0;

    // sort-based relabel
    bool sr_bufs = false;
    unsigned long long* d_sr_keys[2] = {nullptr, nullptr};
    uint32_t* d_sr_perm[2] = {nullptr, nullptr};
    uint32_t* d_sr_head = nullptr;
    uint32_t* d_sr_gstart = nullptr;
    void* d_sr_tmp = nullptr;
    size_t sr_tmp_bytes = 0;

    // device-side round loop
    cudaGraph_t loop_graph = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    int loop_relabel = -1;
    int loop_no_persist = -1;
    int loop_persist_log2 = -2;
    int loop_grid_per_sm = -1;
    float first_sig_ms = 0.f;       // the last refinement's first signature kernel
    uint64_t first_sig_arcs = 0;
    uint64_t body_kernels = 0;  // kernels in one iteration of the captured loop
    bool oneshot = false;       // refined once and freed (rbsc_refine): capturing and
                                // instantiating the loop graph would cost more than it saves

    // arcs kept in host memory (rbsc_graph_upload_streamed): d_idx / d_wt are
    // device-accessible views of page-locked host arrays; a signature pass
    // over them copies chunks of tiles into d_chunk on copy_stream
    bool host_arcs = false;
    bool arcs_on_host = false;      // the active set still uses the host arcs
    void* reg_idx = nullptr;        // host ranges page-locked here, released at free
    void* reg_wt = nullptr;
    uint32_t chunk_tiles = 0;
    uint32_t* d_chunk[2] = {nullptr, nullptr};
    uint64_t* d_chunk_wt[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};
    cudaEvent_t ev_used[2] = {nullptr, nullptr};
    uint64_t resident_cap = 0;      // arcs the compacted (device) arc sets hold
    uint64_t streamed_bytes = 0;    // copied by the streamed passes of the last refinement
    uint32_t streamed_passes = 0;
    // one-shot upload that overlaps the refinement: the heads arrive in
    // chunks (copied into d_idx on copy_stream) during the first pass that
    // reads them; until then d_idx is only partly filled
    bool stream_upload = false;
    const uint32_t* h_upload = nullptr;
    // the one-shot call's host colours, already copied into d_init by the load
    const uint32_t* h_init_loaded = nullptr;
    // a page-locked source: every chunk's copy is issued when the graph is
    // loaded, so the host link stays busy through the set-up kernels and the
    // initial pass; chunk c's copy completes ev_chunk[c]
    bool upload_issued = false;
    static constexpr int kUploadChunks = 8;
    cudaEvent_t ev_chunk[kUploadChunks] = {};
};

rbsc_status rbsc_fail(rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...);
rbsc_status rbsc_cuda_fail(rbsc_ctx* ctx, cudaError_t e, const char* what, int line);
rbsc_status dev_alloc(rbsc_ctx* ctx, void** p, size_t bytes);
void dev_free(rbsc_ctx* ctx, void*& p);
rbsc_status host_alloc(rbsc_ctx* ctx, void** p, size_t bytes);
void host_free(rbsc_ctx* ctx, void*& p);
rbsc_status ensure_temp(rbsc_ctx* ctx, rbsc_graph* g, size_t bytes);
rbsc_status graph_prepare(rbsc_ctx* ctx, rbsc_graph* g);
rbsc_status graph_alloc_csr(rbsc_ctx* ctx, rbsc_graph* g, bool weighted);
rbsc_status refine_resident(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init, uint32_t* d_out, rbsc_stats* stats,
                            rbsc_kernel_times* kt);

// Device scratch of one call: every block is released when it goes out of
// scope (the modules that build their own working set per call).
struct Scratch {
    rbsc_ctx* ctx;
    std::vector<void*> blocks;
    explicit Scratch(rbsc_ctx* c) : ctx(c) {}
    ~Scratch()
    {
        for (void*& b : blocks) dev_free(ctx, b);
    }
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    template <typename T> rbsc_status get(T** p, size_t count)
    {
        void* b = nullptr;
        const rbsc_status st = dev_alloc(ctx, &b, std::max<size_t>(count, 1) * sizeof(T));
        if (st != RBSC_OK) return st;
        blocks.push_back(b);
        *p = static_cast<T*>(b);
        return RBSC_OK;
    }
    void release(void* p)
    {
        for (void*& b : blocks)
            if (b == p) dev_free(ctx, b);
    }
};

// Status propagation inside functions that have a `ctx` in scope.
#define EK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return rbsc_cuda_fail(ctx, e_, #call, __LINE__); \
    } while (0)
#define EKS(call)                      \
    do {                               \
        rbsc_status s_ = (call);       \
        if (s_ != RBSC_OK) return s_;  \
    } while (0)

// sort-based relabel (sortrelabel.cu)
rbsc_status ensure_sort_relabel_bufs(rbsc_ctx* ctx, rbsc_graph* g);
rbsc_status launch_sort_relabel(rbsc_ctx* ctx, rbsc_graph* g, cudaStream_t s);
void sortrelabel_release(rbsc_graph* g);
