// rbsc_driver.cu -- builds the reference GPU program src/rbsc/rbsc.cu,
// UNMODIFIED, with its standard input served from memory.
//
// TEST INFRASTRUCTURE ONLY (it is the checker and the measured competitor,
// never the product).
//
// The reference reads its arcs-cuda text one getchar() at a time
// (rbsc.cu:156-180), and glibc's getchar takes the stdin lock on every call:
// a multi-GB graph then spends minutes in parsing, outside the program's own
// timer (rbsc.cu:272, 489-494) but inside the wall time of a run.  Here the
// whole input is read first and getchar is redirected, for the reference
// translation unit only, to a function serving the captured bytes.  Nothing
// else changes: the refinement, its timer and its three output lines are the
// reference's own.  oracle/Makefile passes -I<reference>/src/rbsc.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdio.h>
#include <stdlib.h>
#include <string>

static std::string g_in;
static size_t g_pos = 0;

static int hook_getchar() { return g_pos < g_in.size() ? (unsigned char)g_in[g_pos++] : EOF; }

#define main ref_rbsc_main
#define getchar hook_getchar
#include "rbsc.cu"
#undef main
#undef getchar

int main(int argc, char** argv)
{
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, stdin)) > 0) g_in.append(buf, k);
    if (g_in.empty() || g_in.back() != '\n') g_in.push_back('\n');
    return ref_rbsc_main(argc, argv);
}
