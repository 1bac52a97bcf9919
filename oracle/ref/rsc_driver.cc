// rsc_driver.cc -- builds the reference CPU program src/rsc/rsc.cpp,
// UNMODIFIED, into a binary that also reports what the reference computes but
// does not print: its final partition and its round count.
//
// TEST INFRASTRUCTURE ONLY (it is the checker, never the product).
//
// The reference source is #included from the reference tree at compile time
// (oracle/Makefile passes -I<reference>/src/rsc); no reference code is copied
// into this repository.  The preprocessor redirects five names, for the
// reference translation unit only:
//   main      -> ref_rsc_main   called from this file's main()
//   getchar   -> hook_getchar   serves the stdin text captured up front
//   malloc    -> hook_malloc    records the reference's arrays; the 4th block
//                               allocated by rsc.cpp:111 is w, the colouring
//   printf    -> hook_printf    captures the three result lines (rsc.cpp:148-150)
//   std::sort -> std::hook_sort counts rounds: rsc.cpp:130 sorts once per round
//
// Output (stdout):   the three captured lines, then "rounds R", then
//                    "round_s d1 .. d{R-1}", then
//                    "labels l0 l1 ... l{n-1}" (w after the last round).
//
// round_s: the steady-clock time between successive entries of the sort of
// rsc.cpp:130, i.e. one complete round each (sort, gather, sum, reorder of
// one round, then spmv and make_indexes of the next).
//
// Options:
//   --runs K     parse the input once, then run the refinement K times: at the
//                first allocation after parsing (w, rsc.cpp:111) the process
//                forks one child per run, in turn; each child carries out the
//                rest of rsc's main (its own timer, rsc.cpp:116-147) and
//                prints its own block of lines.  The parsed arrays are shared
//                copy-on-write and never written by the refinement.
//   --round-samples S
//                as --runs, but fork runs until they have reported at least S
//                round_s values in all (at most 1000 runs); the children add
//                their counts to a shared page.
//   --no-labels  omit the labels line.
#include <stdio.h>
#include <sys/mman.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>
#include <stdlib.h>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

static std::string g_in;
static size_t g_pos = 0;
static std::vector<void*> g_blocks;
static std::vector<size_t> g_sizes;
static std::string g_out;
static unsigned g_sorts = 0;
static std::vector<std::chrono::steady_clock::time_point> g_sort_at;
static int g_runs = 1;
static long g_round_samples = 0;
static long* g_samples_seen = nullptr;  // shared with the children (MAP_SHARED)
static bool g_child = false;

static void fork_runs();

static int hook_getchar() { return g_pos < g_in.size() ? (unsigned char)g_in[g_pos++] : EOF; }
static void* hook_malloc(size_t n)
{
    void* p = std::malloc(n);
    g_blocks.push_back(p);
    g_sizes.push_back(n);
    if (g_blocks.size() == 4 && (g_runs > 1 || g_round_samples > 0) && !g_child) fork_runs();
    return p;
}
static int hook_printf(const char* fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    int k = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_out += buf;
    return k;
}
namespace std {
template <class It, class Cmp> void hook_sort(It a, It b, Cmp c)
{
    ++g_sorts;
    g_sort_at.push_back(std::chrono::steady_clock::now());
    std::sort(a, b, c);
}
}

#define main ref_rsc_main
#define getchar hook_getchar
#define malloc hook_malloc
#define printf hook_printf
#define sort hook_sort
#include "rsc.cpp"
#undef main
#undef getchar
#undef malloc
#undef printf
#undef sort

static bool g_labels = true;

// In the parent: one child per run, one after another; the parent itself
// never returns into rsc's main.
static void fork_runs()
{
    if (g_round_samples > 0) {
        void* p = mmap(nullptr, sizeof(long), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) std::_Exit(6);
        g_samples_seen = static_cast<long*>(p);
        *g_samples_seen = 0;
        g_runs = 1000;
    }
    for (int r = 0; r < g_runs; ++r) {
        if (g_samples_seen && *g_samples_seen >= g_round_samples) break;
        std::fflush(stdout);
        const pid_t pid = fork();
        if (pid < 0) std::_Exit(4);
        if (pid == 0) {
            g_child = true;
            return;
        }
        int st = 0;
        if (waitpid(pid, &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) std::_Exit(5);
    }
    std::fflush(stdout);
    std::_Exit(0);
}

int main(int argc, char** argv)
{
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--runs") && i + 1 < argc) g_runs = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--round-samples") && i + 1 < argc) g_round_samples = std::atol(argv[++i]);
        else if (!std::strcmp(argv[i], "--no-labels")) g_labels = false;
    }
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, stdin)) > 0) g_in.append(buf, k);
    if (g_in.empty() || g_in.back() != '\n') g_in.push_back('\n');
    int rc = ref_rsc_main();
    fputs(g_out.c_str(), stdout);
    if (rc != 0) return rc;
    std::printf("rounds %u\n", g_sorts);
    std::string rl = "round_s";
    for (size_t i = 1; i < g_sort_at.size(); ++i) {
        char t[32];
        std::snprintf(t, sizeof t, " %.6f", std::chrono::duration<double>(g_sort_at[i] - g_sort_at[i - 1]).count());
        rl += t;
    }
    rl += '\n';
    fputs(rl.c_str(), stdout);
    if (g_samples_seen && g_sort_at.size() > 1) *g_samples_seen += (long)(g_sort_at.size() - 1);
    if (!g_labels) {
        std::fflush(stdout);
        return 0;
    }
    if (g_blocks.size() < 4) return 3;
    const uint64_t* w = (const uint64_t*)g_blocks[3];
    size_t n = g_sizes[3] / sizeof(uint64_t);
    std::string line = "labels";
    for (size_t i = 0; i < n; ++i) { line += ' '; line += std::to_string(w[i]); }
    line += '\n';
    fputs(line.c_str(), stdout);
    return 0;
}
