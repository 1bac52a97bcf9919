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
//                    "labels l0 l1 ... l{n-1}" (w after the last round).
#include <stdio.h>
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

static int hook_getchar() { return g_pos < g_in.size() ? (unsigned char)g_in[g_pos++] : EOF; }
static void* hook_malloc(size_t n)
{
    void* p = std::malloc(n);
    g_blocks.push_back(p);
    g_sizes.push_back(n);
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

int main()
{
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, stdin)) > 0) g_in.append(buf, k);
    if (g_in.empty() || g_in.back() != '\n') g_in.push_back('\n');
    int rc = ref_rsc_main();
    fputs(g_out.c_str(), stdout);
    if (rc != 0) return rc;
    std::printf("rounds %u\n", g_sorts);
    if (g_blocks.size() < 4) return 3;
    const uint64_t* w = (const uint64_t*)g_blocks[3];
    size_t n = g_sizes[3] / sizeof(uint64_t);
    std::string line = "labels";
    for (size_t i = 0; i < n; ++i) { line += ' '; line += std::to_string(w[i]); }
    line += '\n';
    fputs(line.c_str(), stdout);
    return 0;
}
