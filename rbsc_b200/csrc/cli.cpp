// cli.cpp -- the `rbsc` command, with the reference's process surface
// (src/rbsc/rbsc.cu:182-497):
//
//   <arcs-cuda text on stdin> | rbsc [edge_batch_size] [gpus]
//
// stdout: exactly three lines, as rbsc.cu:492-494 prints them -- the
// refinement time in seconds ("%lf"), done (1 = coarsest partition), and the
// number of blocks.  On failure a message goes to stdout and the exit code is
// EXIT_FAILURE, as the reference's CHECK_* macros do (rbsc.cu:15-47).
//
// edge_batch_size: as in the reference.  At least M (or absent): one batch,
// the coarsest partition (done = 1).  Below M: the reference's edge-batch
// (quotient) mode, rbsc.cu:292-487, with the same `done` and `nodes` as the
// reference's program prints (rbsc_refine_edge_batches).  gpus: accepted; one
// process drives one GPU (device 0 unless RBSC_DEVICE is set).
//
// Extra options (after the positional ones):
//   --dump-partition FILE   write the canonical label of every node, one per line
//   --init-colors FILE      initial colours, one uint32 per line (N lines);
//                           refines exactly in one batch
//   --stats                 print a JSON line with rounds and timings to stderr
//   --relabel sort|hash     relabel strategy (default hash)
//   --aggressive            the stop test of the reference's rbsc_aggressive
//                           program (rbsc_aggressive.cu:487) in edge-batch mode
//   --exact                 the coarsest partition whatever edge_batch_size is
//   --csr-cache FILE        read the graph from this binary CSR cache when it
//                           exists (stdin is not read); otherwise parse stdin
//                           and write the cache
//   --bv BASENAME           read the graph from BV (WebGraph) files
//                           BASENAME.properties / .graph / .offsets (BASENAME
//                           or BASENAME.graph may be given) instead of
//                           stdin: the step the reference leaves to webgraph-rs
//                           (its arcs-cuda output, unit weights); with
//                           --csr-cache, the cache is written from it
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/rbsc.h"

// Reads the whole stream; a regular file (stdin redirected from a file) is
// read straight into a buffer of its size, a pipe in 4 MiB blocks.
static bool read_all(FILE* f, std::string& s)
{
    struct stat st;
    if (fstat(fileno(f), &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) s.reserve((size_t)st.st_size + 1);
    std::vector<char> buf((size_t)1 << 22);
    size_t k;
    while ((k = fread(buf.data(), 1, buf.size(), f)) > 0) s.append(buf.data(), k);
    return !ferror(f);
}

int main(int argc, char** argv)
{
    const char* dump = nullptr;
    const char* init_path = nullptr;
    const char* cache_path = nullptr;
    const char* bv_path = nullptr;
    bool want_stats = false, aggressive = false, exact = false;
    int relabel = RBSC_RELABEL_HASH;
    std::vector<const char*> pos;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--dump-partition") && i + 1 < argc) dump = argv[++i];
        else if (!std::strcmp(argv[i], "--init-colors") && i + 1 < argc) init_path = argv[++i];
        else if (!std::strcmp(argv[i], "--stats")) want_stats = true;
        else if (!std::strcmp(argv[i], "--aggressive")) aggressive = true;
        else if (!std::strcmp(argv[i], "--exact")) exact = true;
        else if (!std::strcmp(argv[i], "--csr-cache") && i + 1 < argc) cache_path = argv[++i];
        else if (!std::strcmp(argv[i], "--bv") && i + 1 < argc) bv_path = argv[++i];
        else if (!std::strcmp(argv[i], "--relabel") && i + 1 < argc) relabel = !std::strcmp(argv[++i], "sort") ? RBSC_RELABEL_SORT : RBSC_RELABEL_HASH;
        else pos.push_back(argv[i]);
    }
    // positional arguments, as rbsc.cu:204-205 reads them
    unsigned long long edge_batch = pos.size() >= 1 ? std::strtoull(pos[0], nullptr, 10) : 0;
    unsigned long long gpus = pos.size() >= 2 ? std::strtoull(pos[1], nullptr, 10) : 1;
    (void)gpus;

    rbsc_host_graph hg;
    FILE* cached = cache_path ? std::fopen(cache_path, "rb") : nullptr;
    if (cached) {
        std::fclose(cached);
        if (rbsc_csr_load(cache_path, &hg) != RBSC_OK) {
            std::printf("input error: %s\n", rbsc_last_error(nullptr));
            return EXIT_FAILURE;
        }
    } else {
        if (bv_path) {
            // the basename, or the path of its .graph file
            std::string base(bv_path);
            if (base.size() > 6 && base.compare(base.size() - 6, 6, ".graph") == 0) base.resize(base.size() - 6);
            if (rbsc_bv_load(base.c_str(), &hg, nullptr) != RBSC_OK) {
                std::printf("input error: %s\n", rbsc_last_error(nullptr));
                return EXIT_FAILURE;
            }
        } else {
            std::string text;
            if (!read_all(stdin, text)) {
                std::printf("failed to read standard input\n");
                return EXIT_FAILURE;
            }
            if (rbsc_parse_arcs(text.data(), text.size(), &hg) != RBSC_OK) {
                std::printf("input error: %s\n", rbsc_last_error(nullptr));
                return EXIT_FAILURE;
            }
        }
        if (cache_path) {
            rbsc_csr c{hg.n, hg.m, hg.offsets, 8, hg.indices, hg.weights};
            if (rbsc_csr_save(cache_path, &c) != RBSC_OK) {
                std::printf("cache error: %s\n", rbsc_last_error(nullptr));
                return EXIT_FAILURE;
            }
        }
    }

    std::vector<uint32_t> init;
    if (init_path) {
        FILE* f = std::fopen(init_path, "r");
        if (!f) {
            std::printf("cannot open %s\n", init_path);
            return EXIT_FAILURE;
        }
        unsigned long v;
        while (std::fscanf(f, "%lu", &v) == 1) init.push_back((uint32_t)v);
        std::fclose(f);
        if (init.size() != hg.n) {
            std::printf("%s: expected %u colours, read %zu\n", init_path, hg.n, init.size());
            return EXIT_FAILURE;
        }
    }

    const char* dev_env = std::getenv("RBSC_DEVICE");
    rbsc_opts opts;
    rbsc_opts_default(&opts);
    opts.relabel = relabel;
    rbsc_ctx* ctx = rbsc_ctx_create(dev_env ? std::atoi(dev_env) : 0, &opts);
    if (!ctx) {
        std::printf("CUDA setup failed: %s\n", rbsc_last_error(nullptr));
        return EXIT_FAILURE;
    }
    rbsc_csr csr;
    csr.n = hg.n;
    csr.m = hg.m;
    csr.offsets = hg.offsets;
    csr.offset_bytes = 8;
    csr.indices = hg.indices;
    csr.weights = hg.weights;
    std::vector<uint32_t> labels(hg.n);
    rbsc_stats st;
    const bool batched = !exact && init.empty() && edge_batch > 0 && edge_batch < hg.m;
    rbsc_status rc = batched ? rbsc_refine_edge_batches(ctx, &csr, edge_batch, aggressive ? 1 : 0,
                                                        hg.n ? labels.data() : nullptr, &st, nullptr)
                             : rbsc_refine(ctx, &csr, init.empty() ? nullptr : init.data(), hg.n ? labels.data() : nullptr, &st);
    if (rc != RBSC_OK) {
        std::printf("refinement failed: %s\n", rbsc_last_error(ctx));
        rbsc_ctx_destroy(ctx);
        return EXIT_FAILURE;
    }
    std::printf("%lf\n", st.time_s);
    std::printf("%u\n", st.done);
    std::printf("%lu\n", (unsigned long)st.blocks);
    if (want_stats)
        std::fprintf(stderr,
                     "{\"rounds\": %u, \"blocks\": %u, \"initial_blocks\": %u, \"verified\": %u, \"repairs\": %u, "
                     "\"device_ms\": %.4f, \"verify_ms\": %.4f, \"h2d_ms\": %.4f, \"d2h_ms\": %.4f, \"time_s\": %.6f}\n",
                     st.rounds, st.blocks, st.initial_blocks, st.verified, st.repairs, st.device_ms, st.verify_ms, st.h2d_ms,
                     st.d2h_ms, st.time_s);
    if (dump) {
        FILE* f = std::fopen(dump, "w");
        if (!f) {
            std::printf("cannot write %s\n", dump);
            rbsc_ctx_destroy(ctx);
            return EXIT_FAILURE;
        }
        for (uint32_t i = 0; i < hg.n; ++i) std::fprintf(f, "%u\n", labels[i]);
        std::fclose(f);
    }
    rbsc_ctx_destroy(ctx);
    rbsc_host_graph_free(&hg);
    return 0;
}
