/*
 * rbsc.h -- C ABI of librbsc, a B200 (sm_100a) implementation of rbsc's
 * colour-refinement hot path: the coarsest backward-equivalence (lumpable)
 * partition of a weighted directed graph, i.e. 1-WL colour refinement over
 * successor multisets.
 *
 * The reference exposes this path only as a process (src/rbsc/rbsc.cu:182-497:
 * arcs-cuda text on stdin, `rbsc [edge_batch_size] [gpus]`, three lines on
 * stdout).  The entry points below are what that process is made of, split at
 * the places a caller binding the path through an FFI needs; each one names
 * the part of the reference it replaces.  The `rbsc` CLI built from
 * rbsc_b200/csrc/cli.cpp keeps the reference's process surface on top of them.
 *
 * Conventions
 *   - Plain C types only; no exceptions cross the ABI.
 *   - Every call that can fail returns an rbsc_status (0 = OK, < 0 = error);
 *     rbsc_last_error(ctx) gives the message of the last failure on that
 *     context (ctx may be NULL for failures of rbsc_ctx_create).
 *   - Host pointers are owned by the caller.  Device memory is owned by the
 *     library (per context / per graph) unless a function says otherwise.
 *   - A context is used by one host thread at a time; different contexts may
 *     be used concurrently.
 *   - Graph: N nodes (N < 2^31), M arcs, CSR where row u lists the heads v of
 *     the arcs (u, wt, v) -- the reference's arcs grouped by their start
 *     (rbsc.cu:168-180 requires that grouping).  Weights are optional uint64
 *     (absent = 1), summed modulo 2^64 (rbsc.cu:173, 80-87).
 *   - Output labels are canonical: each node carries the smallest node id of
 *     its block.
 */
#ifndef RBSC_H
#define RBSC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBSC_ABI_VERSION 1

typedef int32_t rbsc_status;
#define RBSC_OK 0
#define RBSC_ERR_INVALID (-1)        /* bad argument / malformed graph           */
#define RBSC_ERR_CUDA (-2)           /* a CUDA runtime call failed               */
#define RBSC_ERR_OOM (-3)            /* device or pinned memory exhausted        */
#define RBSC_ERR_NOT_CONVERGED (-4)  /* max_rounds passes without a fixpoint     */
#define RBSC_ERR_DEVICE (-5)         /* a kernel reported an error flag          */
#define RBSC_ERR_PARSE (-6)          /* malformed arcs-cuda text                 */
#define RBSC_ERR_TOO_LARGE (-7)      /* N >= 2^31 or a size beyond a stated limit */
#define RBSC_ERR_BUSY (-8)           /* serving: admission queue full            */

typedef struct rbsc_ctx rbsc_ctx;
typedef struct rbsc_graph rbsc_graph;

/* Relabel strategies for the per-round "(old colour, signature) -> new colour"
 * step (reference: the two radix sorts + scan of rbsc.cu:384-396). */
#define RBSC_RELABEL_HASH 0   /* lock-free hash table, one probe per node (default) */
#define RBSC_RELABEL_SORT 1   /* hand-written LSD radix sort of (colour, signature, node) */

typedef struct {
    int32_t relabel;          /* RBSC_RELABEL_*                                          */
    int32_t verify;           /* 1 (default): exact collision check at every fixpoint   */
    uint32_t max_rounds;      /* 0 = no limit beyond N + 1                               */
    int32_t use_graph;        /* 1 (default): round loop as one CUDA graph with a
                                 device-side while node; 0 = host-driven loop           */
    uint64_t seed;            /* hash salt seed                                          */
    int32_t test_hash_bits;   /* TEST HOOK: keep only the low k bits of every signature
                                 (0 = off; k < 0 or k >= 64: drop signatures entirely, so
                                 the hashed rounds never split and every split comes
                                 from the exact check and repair).  Forces collisions so
                                 the exact check and repair path can be exercised.      */
    int32_t no_persist;       /* 1: never hand small active sets to the persistent
                                 kernel (every pass stays one launch per phase)         */
    int32_t persist_log2;     /* the persistent kernel takes over once the active arcs
                                 and listed nodes are both <= 2^persist_log2
                                 (0 = default 22)                                       */
    int32_t grid_per_sm;      /* blocks per SM of the pass kernels' grids (0 = 16)      */
    int32_t sig_kernel;       /* signature kernel over device arcs: 0 = default (hot
                                 heads where they apply, by tensor copies (4) when the
                                 driver makes their tensor map, else plain loads), 1 = plain
                                 loads, 2 = staged (each warp's tiles copied to shared
                                 memory by cp.async.bulk; unweighted), 3 = hot heads:
                                 the first pass of a resident graph with >= 2^22 arcs
                                 and <= 256 initial classes reads the class ranks of
                                 the most pointed-to nodes from shared memory, 4 = hot
                                 heads with each warp's tile of heads brought into
                                 shared memory by the tensor memory accelerator
                                 (128-byte swizzled boxes)                              */
    int32_t hot_log2;         /* hot heads: at most 2^hot_log2 nodes, those with the
                                 most in-arcs (0 = default 17; 10..17)                  */
    int32_t persist_bps;      /* blocks of 256 threads per SM of the persistent tail
                                 kernel (0 = as many as fit)                            */
    int32_t persist_sig;      /* signature phase of the persistent tail kernel: 0 = by
                                 the active rows' mean length (one row per lane for
                                 short rows, 4 blocks per SM; 512-arc tiles per warp
                                 otherwise, 3 blocks per SM), 1 = rows, 2 = tiles      */
} rbsc_opts;

typedef struct {
    uint32_t rounds;          /* signature passes until the block count stopped
                                 changing (count before pass 1 = #distinct initial
                                 colours; rbsc.cu:339, 354-425)                         */
    uint32_t blocks;          /* blocks of the final partition (rbsc.cu:494 "nodes")   */
    uint32_t done;            /* 1 = coarsest partition (rbsc.cu:493)                   */
    uint32_t verified;        /* 1 = the exact stability check passed                   */
    uint32_t repairs;         /* exact-check failures that were split and re-refined   */
    uint32_t initial_blocks;  /* distinct initial colours                               */
    double time_s;            /* wall time of the call, as rbsc.cu:272-490 measures it */
    double device_ms;         /* device time of the refinement (CUDA events)            */
    double verify_ms;         /* device time of the exact check(s)                       */
    double h2d_ms;            /* host->device copies inside the call                    */
    double d2h_ms;            /* device->host copies inside the call                    */
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint32_t round_blocks[64];/* block count before pass 1 and after passes 1..63       */
    uint64_t kernel_launches; /* kernels of this library launched by the call            */
    double init_ms;           /* device time: initial colours + active-set setup          */
    double loop_ms;           /* device time: the signature passes (all rounds)          */
    double first_signature_ms;   /* k_signature of the first pass, when launched from the
                                    host (few initial classes), else 0                    */
    uint64_t first_signature_arcs; /* arcs that launch processed                         */
    uint64_t streamed_bytes;  /* host->device bytes of the streamed signature passes
                                 (graphs from rbsc_graph_upload_streamed)                */
    uint32_t streamed_passes; /* signature passes that streamed the arcs                */
    uint32_t first_signature_hot; /* hot heads the first signature kernel read from shared
                                     memory (0: it gathered every rank from global memory) */
} rbsc_stats;

/* Per-kernel device time of one refinement, measured with CUDA events around
 * every launch on the library's stream (host-driven loop, same kernels and
 * same work as the graph-captured loop). */
typedef struct {
    uint32_t passes;          /* hashed passes timed                                     */
    double signature_ms;      /* total over the passes: k_signature                     */
    double insert_ms;         /* table inserts (or the sort-based relabel's sorts)       */
    double relabel_ms;        /* relabel + follower copy                                 */
    double other_ms;          /* table clear, fixpoint test, compaction                  */
    double total_ms;          /* whole refinement, including the exact check             */
    double init_ms;           /* initial-colour pass                                     */
    double setup_ms;          /* node list / follower construction                       */
    float pass_ms[32][4];     /* per pass (first 32): signature, insert, relabel, other  */
    uint64_t pass_arcs[32];   /* arcs in the signature pass                              */
    uint32_t pass_nodes[32];  /* nodes in the relabel list                               */
    double persist_ms;        /* the persistent kernel (small active sets), all its passes */
    uint32_t persist_passes;
} rbsc_kernel_times;

/* A CSR graph.  `offsets` has n+1 entries of `offset_bytes` (4 or 8) bytes;
 * `indices` has m entries; `weights` is NULL or has m entries. */
typedef struct {
    uint32_t n;
    uint64_t m;
    const void* offsets;
    int32_t offset_bytes;
    const uint32_t* indices;
    const uint64_t* weights;
} rbsc_csr;

/* A host CSR owned by the library (filled by the parser and the generators). */
typedef struct {
    uint32_t n;
    uint64_t m;
    uint64_t* offsets;        /* n+1 */
    uint32_t* indices;        /* m   */
    uint64_t* weights;        /* m, or NULL when every weight is 1 */
} rbsc_host_graph;

/* ---- library / context --------------------------------------------------- */

int32_t rbsc_abi_version(void);
void rbsc_opts_default(rbsc_opts* opts);

/* Creates a context on CUDA device `device` (replaces the per-GPU setup of
 * rbsc.cu:234-270).  Returns NULL on failure; see rbsc_last_error(NULL). */
rbsc_ctx* rbsc_ctx_create(int32_t device, const rbsc_opts* opts);
void rbsc_ctx_destroy(rbsc_ctx* ctx);
/* A context keeps the device and pinned buffers of freed graphs and
 * one-shot refinements and hands them out again (no reference counterpart:
 * the reference allocates per run).  rbsc_ctx_trim gives the unused ones
 * back to CUDA; rbsc_ctx_destroy does so too. */
void rbsc_ctx_trim(rbsc_ctx* ctx);
const char* rbsc_last_error(const rbsc_ctx* ctx);
rbsc_status rbsc_ctx_set_opts(rbsc_ctx* ctx, const rbsc_opts* opts);

/* ---- one-shot refinement (the reference's whole single-batch path) -------- */

/* Refines a host CSR: copies it to the device, refines to the fixpoint,
 * checks the result exactly, copies the labels back.  Replaces rbsc.cu:341-445
 * (H2D, round loop, D2H, host relabel) for edge_batch_size >= M.
 * init_colors: NULL (one initial block) or n uint32 colours (any values).
 * out_labels: NULL or n uint32 (canonical labels).  stats: NULL or filled. */
rbsc_status rbsc_refine(rbsc_ctx* ctx, const rbsc_csr* host_graph, const uint32_t* init_colors,
                        uint32_t* out_labels, rbsc_stats* stats);

/* ---- resident graphs ---------------------------------------------------- */

/* Copies a host CSR to the device and builds the per-graph tiling once
 * (replaces rbsc.cu:341-344 and the per-batch setup of 345-352). */
rbsc_status rbsc_graph_upload(rbsc_ctx* ctx, const rbsc_csr* host_graph, rbsc_graph** out);
/* Same from a CSR already in device memory (pointers into this context's
 * device); the arrays are copied, the caller keeps ownership of its own. */
rbsc_status rbsc_graph_from_device(rbsc_ctx* ctx, const rbsc_csr* device_graph, rbsc_graph** out);
/* A resident graph whose arcs stay in host memory: for graphs whose arcs do
 * not fit (or should not live in) device memory.  Offsets, the per-row tiling
 * and all refinement state live on the device; a signature pass over the full
 * arc set streams the heads (and weights) in batches of batch_arcs arcs (0 = a
 * quarter of M) through two device buffers, copying the next batch on a side
 * stream while the signature kernel reads the current one.  Once the arcs of
 * non-singleton rows fit resident_arcs (0 = min(M, 2^31)) they are compacted
 * into device memory and later passes run from there.  The exact check and the
 * compaction read the host arrays directly (mapped page-locked memory).  The
 * caller's indices / weights must stay valid and unchanged while the graph
 * exists; pageable arrays are page-locked here (cudaHostRegister) for its
 * lifetime.  No reference counterpart: the reference's batches
 * (rbsc.cu:302-345) change the result; this mode is exact. */
rbsc_status rbsc_graph_upload_streamed(rbsc_ctx* ctx, const rbsc_csr* host_graph, uint64_t batch_arcs,
                                       uint64_t resident_arcs, rbsc_graph** out);
void rbsc_graph_free(rbsc_graph* g);
rbsc_status rbsc_graph_info(const rbsc_graph* g, uint32_t* n, uint64_t* m);
/* Device pointers of the resident CSR (offsets are uint64). */
rbsc_status rbsc_graph_device_csr(const rbsc_graph* g, const uint64_t** d_offsets,
                                  const uint32_t** d_indices);

/* Refines a resident graph; init/out are HOST pointers (either may be NULL). */
rbsc_status rbsc_graph_refine(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* init_colors,
                              uint32_t* out_labels, rbsc_stats* stats);
/* Refines a resident graph; init/out are DEVICE pointers (either may be NULL).
 * No host<->device copies of graph-sized data happen inside this call. */
rbsc_status rbsc_graph_refine_device(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init_colors,
                                     uint32_t* d_out_labels, rbsc_stats* stats);
/* Measurement entry point (no counterpart in the reference, which times the
 * whole run with std::chrono, rbsc.cu:272, 489-490): refines like
 * rbsc_graph_refine_device, with CUDA events around every kernel launch. */
rbsc_status rbsc_graph_profile(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init_colors,
                               rbsc_kernel_times* times, rbsc_stats* stats);
/* Initial colours floor(log2(out_degree + 1)) written to d_colors (n uint32),
 * computed on the device from the resident offsets. */
rbsc_status rbsc_graph_degree_colors(rbsc_ctx* ctx, rbsc_graph* g, uint32_t* d_colors);

/* ---- the reference's edge-batch (quotient) mode ----------------------------
 * rbsc.cu:292-487 (rbsc_aggressive.cu:487 with `aggressive`): when the arcs do
 * not fit one batch of edge_batch_size arcs, the reference refines each batch
 * of arcs on its own (its sources in one block, arc-less nodes of batch 0 in
 * another, every other node alone), gives every batch class a global id,
 * replaces the graph by its quotient (one representative run per class, heads
 * renamed, parallel arcs merged with summed weights) and repeats until one
 * batch holds all arcs (the coarsest partition: done = 1) or the node count
 * stops shrinking (done = 0, a partition finer than the coarsest one).  This
 * entry point reproduces that mode: the same `nodes` and `done` as the
 * reference's program for the same edge_batch_size, every batch refined
 * exactly on the device.  edge_batch_size 0 = all arcs (one batch).
 * init colours are not part of this mode (the reference has none).
 * out_labels (host, n uint32, may be NULL): canonical labels of the final
 * partition of the input nodes.  stats->blocks = the "nodes" line,
 * stats->done, stats->time_s (wall), stats->rounds = passes of all batch
 * refinements. */
typedef struct {
    uint32_t iterations;      /* outer (quotient) iterations                         */
    uint32_t last_batches;    /* batches of the last iteration                       */
    uint64_t batches_total;   /* batches over all iterations                         */
    uint64_t local_refinements; /* batches that were refined (non-empty after trimming) */
    uint64_t last_arcs;       /* arcs of the last quotient graph                      */
} rbsc_edge_batch_info;

rbsc_status rbsc_refine_edge_batches(rbsc_ctx* ctx, const rbsc_csr* host_graph, uint64_t edge_batch_size,
                                     int32_t aggressive, uint32_t* out_labels, rbsc_stats* stats,
                                     rbsc_edge_batch_info* info);

/* ---- lumping with double weights ------------------------------------------
 * Replaces Valmari's minimiser built with MDP_weight_is_double
 * (src/part_ref/MDPmin.cc:37, 107-113; MDP_minimize.cc:567-637): the weight of
 * a node into a block is the double sum of its arcs' weights into the block,
 * taken in arc order and rounded to float (MDP_round_weight); a sum that
 * rounds to zero counts as no arc.  The result is the coarsest partition that
 * refines the initial colours (NULL = one block) and in which the members of
 * every block have equal rounded sums into every block; labels canonical
 * (smallest node id per block), checked exactly before they are returned.
 * host_graph->weights must be NULL: `weights` (host, m doubles, finite, of
 * magnitude below 2^960) replaces it; m < 2^32, n <= 2^31.  stats: rounds (passes until
 * the block count stopped changing), blocks, verified, repairs, device_ms,
 * round_blocks, kernel_launches.  The minimiser adds a block's weights in
 * the order of the block's members: its float can differ from this one's
 * only when the two double sums fall on different sides of a float rounding
 * boundary. */
rbsc_status rbsc_refine_f64(rbsc_ctx* ctx, const rbsc_csr* host_graph, const double* weights,
                            const uint32_t* init_colors, uint32_t* out_labels, rbsc_stats* stats);

/* ---- autotuning (no reference counterpart) --------------------------------
 * Times refinements of a resident graph (d_init_colors: device colours or
 * NULL) under every combination of the candidate knobs below and returns the
 * fastest as options (rbsc_ctx_set_opts applies them).  Every candidate must
 * give the same blocks and rounds as the context's current options; a
 * candidate that does not is reported as failed and never chosen.  A zero or
 * empty list keeps the context's current value for that knob. */
#define RBSC_TUNE_MAX 8
typedef struct {
    int32_t persist_log2[RBSC_TUNE_MAX];  /* hand-off thresholds to try (-1 = never hand off) */
    uint32_t n_persist;
    int32_t grid_per_sm[RBSC_TUNE_MAX];
    uint32_t n_grid;
    int32_t relabel[RBSC_TUNE_MAX];       /* RBSC_RELABEL_HASH / _SORT                      */
    uint32_t n_relabel;
    int32_t use_graph[RBSC_TUNE_MAX];     /* CUDA-graph loop 1 / host loop 0                */
    uint32_t n_use_graph;
    int32_t sig_kernel[RBSC_TUNE_MAX];    /* signature kernels to try (1 plain, 2 staged,
                                             3 hot heads, 4 hot heads by tensor copies) */
    uint32_t n_sig_kernel;
    uint32_t reps;                        /* timed refinements per candidate (0 = 3)         */
} rbsc_tune_space;

typedef struct {
    uint32_t candidates;      /* combinations timed                                   */
    uint32_t failed;          /* candidates whose result differed (never chosen)      */
    double best_ms;           /* median device time of the chosen candidate           */
    double default_ms;        /* median device time under the context's options       */
    double ms[64];            /* median device time of candidate i (first 64)         */
    rbsc_opts opts[64];       /* the options of candidate i (first 64)               */
} rbsc_tune_report;

void rbsc_tune_space_default(rbsc_tune_space* space);
rbsc_status rbsc_graph_autotune(rbsc_ctx* ctx, rbsc_graph* g, const uint32_t* d_init_colors,
                                const rbsc_tune_space* space, rbsc_opts* best, rbsc_tune_report* report);

/* ---- input formats (reference: read_graph, rbsc.cu:156-180) -------------- */

/* Parses arcs-cuda text ("N\nM\n" + M lines "u wt v", arcs grouped by u;
 * webgraph-rs cli/src/to/arcscuda.rs:61-66) into a host CSR.  Unlike the
 * reference reader it stops at end of input, rejects non-digits, out-of-range
 * node ids, fewer than M arcs and arcs not grouped by source. */
rbsc_status rbsc_parse_arcs(const char* text, size_t len, rbsc_host_graph* out);
void rbsc_host_graph_free(rbsc_host_graph* g);

/* A binary cache of a host CSR (8-byte offsets): rbsc_csr_save writes it,
 * rbsc_csr_load reads it back (checksum, size and offsets checked), so a graph
 * parsed once from text loads again without the parse.  No reference
 * counterpart: the reference parses its text input on every run
 * (rbsc.cu:156-180).  Free with rbsc_host_graph_free. */
rbsc_status rbsc_csr_save(const char* path, const rbsc_csr* host_graph);
rbsc_status rbsc_csr_load(const char* path, rbsc_host_graph* out);

/* Reads a BV-compressed graph (the WebGraph format of the LAW datasets the
 * reference benchmarks on, which its webgraph-rs decodes to arcs-cuda text,
 * cli/src/to/arcscuda.rs:61-66): basename.properties, basename.graph and, if
 * present, basename.offsets (used to check every list's start).  Default
 * codes only (empty compressionflags).  Row u = the successors of u, sorted;
 * no weights.  Free with rbsc_host_graph_free. */
typedef struct {
    uint64_t copied_arcs;     /* successors copied from a referenced list          */
    uint64_t interval_arcs;   /* successors in intervals                           */
    uint64_t residual_arcs;   /* successors coded as gaps                          */
    uint64_t bits;            /* bits of the .graph stream decoded                 */
    uint32_t offsets_checked; /* 1: every list started at its .offsets position     */
    uint32_t pad;
} rbsc_bv_stats;

rbsc_status rbsc_bv_load(const char* basename, rbsc_host_graph* out, rbsc_bv_stats* stats);

/* ---- synthetic workloads (stand-ins for the reference's LAW graphs) ------ */

/* Directed R-MAT: 2^scale nodes, edge_factor * 2^scale generated arcs with
 * quadrant probabilities (a, b, c, 1-a-b-c); duplicates and self-loops removed;
 * rows sorted.  Counter-based: the same (scale, ef, a, b, c, seed) gives the
 * same graph on the host and on the device. */
rbsc_status rbsc_gen_rmat_device(rbsc_ctx* ctx, uint32_t scale, uint32_t edge_factor, double a,
                                 double b, double c, uint64_t seed, rbsc_graph** out);
rbsc_status rbsc_gen_rmat_host(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                               uint64_t seed, int32_t threads, rbsc_host_graph* out);
/* The same graph generated on the device in source buckets (every bucket
 * regenerates the arcs and keeps those whose source falls in it, sorts and
 * deduplicates them) and written to page-locked host memory: for graphs
 * larger than device memory (R-MAT scale 28, edge factor 32: 8.6e9 arcs,
 * 34 GB of heads).  Free with rbsc_host_graph_free_pinned. */
rbsc_status rbsc_gen_rmat_pinned(rbsc_ctx* ctx, uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                 uint64_t seed, rbsc_host_graph* out);
void rbsc_host_graph_free_pinned(rbsc_host_graph* g);

/* Directed Erdos-Renyi G(n, p), p = mean_degree / (n - 1), no self-loops,
 * rows sorted; and its random lift: every node copied `lift` times, every
 * arc (u, v) of a G(base_n, p) base becoming the arcs (u*lift + i,
 * v*lift + pi(i)) for a uniform permutation pi per base arc.  Counter-based:
 * the same arguments give the same graph for any thread count.  Free with
 * rbsc_host_graph_free. */
rbsc_status rbsc_gen_er_host(uint32_t n, double mean_degree, uint64_t seed, int32_t threads, rbsc_host_graph* out);
rbsc_status rbsc_gen_lift_host(uint32_t base_n, double mean_degree, uint32_t lift, uint64_t seed, int32_t threads,
                               rbsc_host_graph* out);

/* ---- batches of small graphs (no reference counterpart) ------------------
 * Many graphs side by side in one CSR over global node ids (no arc between
 * two graphs), graph i owning nodes [graph_nodes[i], graph_nodes[i+1]).  They
 * are refined together, as their disjoint union, so that colours form one
 * namespace shared by all graphs: a colour is the smallest global node id of
 * its class over the whole batch.  Two graphs are told apart by colour
 * refinement (1-WL) iff their colour histograms differ.  Each graph's own
 * partition is the one a refinement of that graph alone gives. */
typedef struct {
    uint32_t num_graphs;
    uint64_t* graph_nodes;    /* num_graphs+1                                          */
    uint32_t* labels;         /* n initial labels                                      */
    rbsc_host_graph csr;      /* the graphs side by side, global node ids               */
} rbsc_graph_batch;

/* Output arrays (host memory, each may be NULL). */
typedef struct {
    uint32_t* colors;         /* n: shared colour of each node                         */
    uint32_t* local;          /* n: smallest local node id of the node's block in its
                                 own graph (the canonical label of a refinement of
                                 that graph alone)                                       */
    uint32_t* blocks;         /* num_graphs: blocks of each graph                       */
    uint64_t* fingerprint;    /* num_graphs: 64-bit digest of the colour histogram      */
    uint64_t* hist_offsets;   /* num_graphs+1: entries of each graph's histogram        */
    uint32_t* hist_colors;    /* up to n: a graph's colours, increasing                 */
    uint32_t* hist_counts;    /* up to n: its nodes of that colour                      */
} rbsc_batch_result;

/* Seeded generator of the small-graph batch: num_graphs graphs with node
 * counts uniform in [nmin, nmax]; even-numbered graphs Erdos-Renyi with edge
 * probability 4/(n-1), odd-numbered random 3-regular (n rounded down to
 * even, at least 4); symmetric arcs; labels uniform in {1..num_labels}.
 * Free with rbsc_graph_batch_free. */
rbsc_status rbsc_gen_wl_batch(uint32_t num_graphs, uint32_t nmin, uint32_t nmax, uint32_t num_labels,
                              uint64_t seed, int32_t threads, rbsc_graph_batch* out);
void rbsc_graph_batch_free(rbsc_graph_batch* b);

/* One-shot batch refinement: host CSR of the batch in, per-graph results out. */
rbsc_status rbsc_batch_refine(rbsc_ctx* ctx, const rbsc_csr* graphs, const uint64_t* graph_nodes,
                              uint32_t num_graphs, const uint32_t* init_colors, rbsc_batch_result* out,
                              rbsc_stats* stats);
/* The same on a resident graph holding the batch (rbsc_graph_upload). */
rbsc_status rbsc_graph_batch_refine(rbsc_ctx* ctx, rbsc_graph* g, const uint64_t* graph_nodes,
                                    uint32_t num_graphs, const uint32_t* init_colors,
                                    rbsc_batch_result* out, rbsc_stats* stats);

/* ---- serving: continuous batching of refinement jobs ---------------------
 * No counterpart in the reference, which refines one graph per process run
 * (rbsc.cu:182-497).  A server owns `slots` executors on one device, each a
 * context with its own stream and host thread, so the jobs of different slots
 * overlap on the GPU.  Jobs are admitted in arrival order as a slot and device
 * memory free up: a job is started only while the estimated device footprint
 * of all running work stays within `hbm_budget` (rbsc_serve_footprint).  When
 * the oldest waiting job is small (at most pack_max_arcs arcs, unweighted),
 * it is started together with the other small jobs waiting behind it, up to
 * pack_max_graphs jobs and pack_arc_budget arcs, as one batch refinement of
 * their disjoint union (rbsc_batch_refine): every job still gets exactly the
 * labels and block count a refinement of its graph alone gives.  With two or
 * more slots, large jobs occupy at most all slots but one while small jobs
 * wait: when every other slot runs a large job, the idle one goes to the
 * oldest small job before the oldest large one.
 *
 * A job's host buffers (CSR, initial colours, output labels) belong to the
 * caller and must stay valid and unchanged until the job's result has been
 * collected by rbsc_serve_poll or rbsc_serve_wait (each result is handed out
 * once).  Every call is thread-safe. */
#define RBSC_PENDING 1               /* serving: the job has not finished yet    */

typedef struct rbsc_server rbsc_server;

typedef struct {
    int32_t device;
    uint32_t slots;           /* executors (contexts / streams / host threads), 0 = 2 */
    uint64_t hbm_budget;      /* bytes of device memory running work may take;
                                 0 = half of the device's free memory at creation     */
    uint64_t pack_max_arcs;   /* jobs of at most this many arcs are packed, 0 = 2^18  */
    uint32_t pack_max_graphs; /* jobs per packed batch, 0 = 4096; 1 = never pack      */
    uint64_t pack_arc_budget; /* arcs (and nodes) per packed batch, 0 = 2^22          */
    uint32_t queue_cap;       /* jobs waiting to start, 0 = 65536; submit beyond
                                 returns RBSC_ERR_BUSY                                */
    rbsc_opts opts;           /* refinement options of every job (no_persist is forced
                                 on: a cooperative grid must not share the GPU with
                                 the other slots' kernels)                            */
    int32_t dry_run;          /* TEST HOOK: 1 = no GPU work at all; each job "runs" for
                                 dry_run_ns_per_arc * arcs + 20 us of host sleep and
                                 writes no labels (exercises admission and packing)   */
    uint32_t dry_run_ns_per_arc;
} rbsc_serve_opts;

typedef struct {
    int32_t status;           /* RBSC_OK or the job's error                            */
    uint32_t blocks;          /* blocks of the job's partition                         */
    uint32_t rounds;          /* passes of the refinement that ran it (for a packed job,
                                 the passes of the whole batch)                        */
    uint32_t packed;          /* jobs in the batch it ran in (1 = alone)               */
    uint32_t slot;            /* executor that ran it                                  */
    uint32_t pad;
    uint64_t footprint;       /* device bytes admitted for its batch                   */
    double queue_ms;          /* submit -> start                                        */
    double service_ms;        /* start -> labels in host memory                          */
    double latency_ms;        /* submit -> finished                                      */
    char error[128];          /* message when status != RBSC_OK                         */
} rbsc_serve_result;

typedef struct {
    uint64_t submitted, completed, failed, rejected;
    uint64_t batches;         /* executions started (packs and single jobs)            */
    uint64_t packed_jobs;     /* jobs that ran inside a pack of two or more            */
    uint64_t queued, running; /* now                                                   */
    uint64_t reserved;        /* admitted footprint of running work, now               */
    uint64_t peak_reserved;   /* its maximum so far                                    */
    uint32_t peak_busy_slots; /* most slots busy at once                               */
    uint32_t slots;
    uint64_t hbm_budget;
} rbsc_serve_stats;

void rbsc_serve_opts_default(rbsc_serve_opts* opts);
/* Device bytes the server reserves for a refinement of `graphs` graphs with n
 * nodes and m arcs in total (an upper estimate of what the refinement
 * allocates). */
uint64_t rbsc_serve_footprint(uint64_t n, uint64_t m, int32_t weighted, uint32_t graphs);
rbsc_status rbsc_serve_create(const rbsc_serve_opts* opts, rbsc_server** out);
/* Finishes the running work, cancels the waiting jobs and frees everything. */
void rbsc_serve_destroy(rbsc_server* srv);
const char* rbsc_serve_last_error(const rbsc_server* srv);
/* Queues a job.  init_colors: NULL or n colours; out_labels: NULL or n uint32
 * (canonical labels).  RBSC_ERR_TOO_LARGE when the job alone exceeds the
 * budget, RBSC_ERR_BUSY when the queue is full. */
rbsc_status rbsc_serve_submit(rbsc_server* srv, const rbsc_csr* host_graph, const uint32_t* init_colors,
                              uint32_t* out_labels, uint64_t* job_id);
/* RBSC_OK (result filled, job released), RBSC_PENDING, or RBSC_ERR_INVALID
 * for an unknown job. */
rbsc_status rbsc_serve_poll(rbsc_server* srv, uint64_t job_id, rbsc_serve_result* result);
/* Like poll, waiting up to timeout_ms (< 0: no limit). */
rbsc_status rbsc_serve_wait(rbsc_server* srv, uint64_t job_id, int64_t timeout_ms, rbsc_serve_result* result);
rbsc_status rbsc_serve_stats_get(rbsc_server* srv, rbsc_serve_stats* stats);

/* ---- refinement without device allocation -------------------------------- */

/* No counterpart in the reference (which allocates everything it uses,
 * rbsc.cu:234-270).  For callers that cannot allocate device memory -- code
 * running while another framework owns the device memory pool, real-time paths
 * that must avoid the device synchronisation an allocation can cause, hosts
 * that only hand out pointers into memory they manage themselves.
 *
 * Refines a small graph held in the caller's device memory in one kernel
 * launch on `stream` (a cudaStream_t, or NULL for the default stream) of the
 * current device.  Limits: N <= RBSC_NOALLOC_MAX_NODES, M <=
 * RBSC_NOALLOC_MAX_ARCS; larger graphs are rejected with RBSC_ERR_TOO_LARGE.
 * d_init_colors (may be NULL), d_out_labels (N uint32, canonical labels) and
 * d_result are device pointers; d_result is written when the kernel ends
 * (status RBSC_OK, RBSC_ERR_NOT_CONVERGED, RBSC_ERR_DEVICE, or RBSC_ERR_INVALID
 * when the kernel's own check of the graph fails: offsets[0] != 0, offsets
 * decreasing, offsets[N] != M, or a head >= N; that check runs before any read
 * indexed by the graph, and d_out_labels is then left untouched).  opts may be
 * NULL (defaults; relabel, verify and use_graph are ignored: the kernel always
 * hashes and checks exactly).  The return value reports argument errors and
 * launch failures only; synchronise the stream before reading d_result.
 *
 * Nothing is allocated: all scratch (about 5 MB) is one static device array of
 * the library, held by every GPU that loads it until the process exits, and
 * shared by all calls -- calls whose kernels overlap on the GPU race on it.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process; make that
 * first call before any stream capture, and do not call this entry point on a
 * device after cudaDeviceReset on it (the kept address may no longer be
 * mapped). */
#define RBSC_NOALLOC_MAX_NODES 16384u
#define RBSC_NOALLOC_MAX_ARCS (1u << 24)

typedef struct {
    uint32_t blocks;
    uint32_t rounds;
    uint32_t repairs;
    int32_t status;
} rbsc_noalloc_result;

rbsc_status rbsc_refine_noalloc(const rbsc_csr* device_graph, const uint32_t* d_init_colors,
                                uint32_t* d_out_labels, rbsc_noalloc_result* d_result,
                                const rbsc_opts* opts, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RBSC_H */
