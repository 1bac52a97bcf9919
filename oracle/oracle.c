/*
 * oracle.c -- CPU restatement of rbsc's colour-refinement path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * path is compared against; nothing in the product (librbsc, the CLI, the
 * Python package) links, loads or calls it.  Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py use it.
 *
 * Parity status: pinned.  Its results are checked against the outputs of the
 * reference programs themselves (src/rsc/rsc.cpp and the Valmari minimiser in
 * src/part_ref, compiled unmodified from their sources by oracle/Makefile) on
 * the fixtures in tests/golden/.
 *
 * Problem (src/part_ref/MDP_minimize.cc:56-64, src/rsc/rsc.cpp:71-144):
 * a graph is a list of weighted arcs (u, wt, v) grouped by u (CSR row u = the
 * arcs whose start is u).  Two nodes are equivalent iff they are in the same
 * block of the current partition and, for every block C, the sums of the
 * weights of their arcs into C are equal.  The result is the coarsest stable
 * refinement of the initial partition (all nodes in one block unless initial
 * colours are given).
 *
 * Two restatements live here:
 *   orc_refine_exact  -- exact refinement: each round every node's signature
 *                        is (old block, sorted list of (successor block,
 *                        summed weight)), compared exactly, never hashed.
 *   orc_refine_rsc    -- the reference CPU program's own randomised loop
 *                        (rsc.cpp:63-144): hashed sums, lexicographic sort of
 *                        (sum, old colour), dense ranks, stop when the block
 *                        count stops changing.
 *
 * Labels returned by both are canonical: every node is labelled with the
 * smallest node id of its block.
 *
 * Round count, "GPU convention" (src/rbsc/rbsc.cu:339, 354-425): rounds =
 * number of signature passes until a pass leaves the block count unchanged,
 * the count before the first pass being the number of distinct initial
 * colours.  rsc.cpp:104-144 starts its count at N instead; orc_refine_rsc
 * reports both.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* index merge sort with a context comparator (stable)                 */
/* ------------------------------------------------------------------ */
typedef int (*orc_cmp_fn)(uint32_t a, uint32_t b, const void* ctx);

static void msort_idx(uint32_t* a, uint32_t* tmp, size_t n, orc_cmp_fn cmp, const void* ctx)
{
    for (size_t width = 1; width < n; width *= 2) {
        for (size_t lo = 0; lo < n; lo += 2 * width) {
            size_t mid = lo + width < n ? lo + width : n;
            size_t hi = lo + 2 * width < n ? lo + 2 * width : n;
            size_t i = lo, j = mid, k = lo;
            while (i < mid && j < hi) {
                if (cmp(a[j], a[i], ctx) < 0) tmp[k++] = a[j++];
                else tmp[k++] = a[i++];
            }
            while (i < mid) tmp[k++] = a[i++];
            while (j < hi) tmp[k++] = a[j++];
        }
        memcpy(a, tmp, n * sizeof(uint32_t));
    }
}

/* ------------------------------------------------------------------ */
/* canonical labels                                                    */
/* ------------------------------------------------------------------ */

/* ctx points at a `const uint32_t*` label array */
static int cmp_lab(uint32_t a, uint32_t b, const void* ctx)
{
    const uint32_t* l = *(const uint32_t* const*)ctx;
    return l[a] < l[b] ? -1 : (l[a] > l[b] ? 1 : 0);
}

/* Relabel an arbitrary labelling so that each block carries the smallest node
 * id in it.  Labels may be any uint32 values.  Returns the number of blocks. */
uint32_t orc_canonicalize(uint32_t n, const uint32_t* in, uint32_t* out)
{
    if (n == 0) return 0;
    uint32_t* ord = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; ++i) ord[i] = i;
    /* sort node ids by label, stable -> first of each run is the minimum */
    const uint32_t* c = in;
    msort_idx(ord, tmp, n, cmp_lab, &c);
    uint32_t blocks = 0, rep = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (i == 0 || in[ord[i]] != in[ord[i - 1]]) { rep = ord[i]; ++blocks; }
        out[ord[i]] = rep;
    }
    free(ord); free(tmp);
    return blocks;
}

/* ------------------------------------------------------------------ */
/* exact refinement                                                    */
/* ------------------------------------------------------------------ */
typedef struct {
    const uint32_t* cur;     /* old labels                               */
    const uint64_t* sstart;  /* per node: start of its compressed list   */
    const uint32_t* slen;    /* per node: number of (label, weight) runs */
    const uint32_t* slab;    /* run labels                               */
    const uint64_t* swt;     /* run weight sums (mod 2^64)               */
} exact_ctx;

static int cmp_exact(uint32_t a, uint32_t b, const void* vctx)
{
    const exact_ctx* c = (const exact_ctx*)vctx;
    if (c->cur[a] != c->cur[b]) return c->cur[a] < c->cur[b] ? -1 : 1;
    if (c->slen[a] != c->slen[b]) return c->slen[a] < c->slen[b] ? -1 : 1;
    const uint32_t* la = c->slab + c->sstart[a];
    const uint32_t* lb = c->slab + c->sstart[b];
    const uint64_t* wa = c->swt + c->sstart[a];
    const uint64_t* wb = c->swt + c->sstart[b];
    for (uint32_t i = 0; i < c->slen[a]; ++i) {
        if (la[i] != lb[i]) return la[i] < lb[i] ? -1 : 1;
        if (wa[i] != wb[i]) return wa[i] < wb[i] ? -1 : 1;
    }
    return 0;
}

typedef struct { uint32_t lab; uint64_t w; } lw_pair;

static int cmp_lw(const void* x, const void* y)
{
    const lw_pair* a = (const lw_pair*)x;
    const lw_pair* b = (const lw_pair*)y;
    return a->lab < b->lab ? -1 : (a->lab > b->lab ? 1 : 0);
}

/*
 * Exact coarsest stable refinement.
 *   off[n+1], idx[m]: CSR (row u = successors of u), wt[m] optional (NULL =
 *   unit weights), init[n] optional initial colours (NULL = one block).
 *   labels_out[n]: canonical labels (min node id per block).
 *   round_blocks (optional, max_rounds+1 entries): block count before the
 *   first pass (index 0) and after every pass.
 * Returns 0, or -1 if max_rounds passes did not reach a fixpoint.
 */
int orc_refine_exact(uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt,
                     const uint32_t* init, uint32_t* labels_out, uint32_t* rounds_out,
                     uint32_t* blocks_out, uint32_t* round_blocks, uint32_t max_rounds)
{
    *rounds_out = 0; *blocks_out = 0;
    if (n == 0) { if (round_blocks) round_blocks[0] = 0; return 0; }
    uint64_t m = off[n];
    uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* nxt = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* ord = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint64_t* sstart = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint32_t* slen = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* slab = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
    uint64_t* swt = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
    lw_pair* row = (lw_pair*)malloc(sizeof(lw_pair) * (m ? m : 1));

    uint32_t prev;
    if (init) prev = orc_canonicalize(n, init, cur);
    else { for (uint32_t i = 0; i < n; ++i) cur[i] = 0; prev = 1; }
    if (round_blocks) round_blocks[0] = prev;

    int status = -1;
    uint32_t r = 0;
    while (r < max_rounds) {
        /* compressed, sorted successor-block lists */
        for (uint32_t u = 0; u < n; ++u) {
            uint64_t b = off[u], e = off[u + 1], d = e - b;
            for (uint64_t k = 0; k < d; ++k) {
                row[k].lab = cur[idx[b + k]];
                row[k].w = wt ? wt[b + k] : 1u;
            }
            qsort(row, (size_t)d, sizeof(lw_pair), cmp_lw);
            uint32_t len = 0;
            sstart[u] = b;
            for (uint64_t k = 0; k < d;) {
                uint32_t lab = row[k].lab;
                uint64_t s = 0;
                while (k < d && row[k].lab == lab) { s += row[k].w; ++k; }
                if (s != 0) { slab[b + len] = lab; swt[b + len] = s; ++len; }
            }
            slen[u] = len;
        }
        exact_ctx c = { cur, sstart, slen, slab, swt };
        for (uint32_t i = 0; i < n; ++i) ord[i] = i;
        msort_idx(ord, tmp, n, cmp_exact, &c);
        uint32_t blocks = 0, rep = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (i == 0 || cmp_exact(ord[i - 1], ord[i], &c) != 0) { rep = ord[i]; ++blocks; }
            nxt[ord[i]] = rep;
        }
        ++r;
        if (round_blocks) round_blocks[r] = blocks;
        uint32_t* sw = cur; cur = nxt; nxt = sw;
        if (blocks == prev) { status = 0; break; }
        prev = blocks;
    }
    memcpy(labels_out, cur, sizeof(uint32_t) * n);
    *rounds_out = r;
    *blocks_out = orc_canonicalize(n, cur, labels_out);
    free(cur); free(nxt); free(ord); free(tmp); free(sstart); free(slen);
    free(slab); free(swt); free(row);
    return status;
}

/* ------------------------------------------------------------------ */
/* exact refinement with double weights                                */
/* ------------------------------------------------------------------ */
typedef struct { uint32_t lab; uint32_t pos; double w; } ld_arc;

/* successor block, then arc position: a stable order of the row */
static int cmp_ld(const void* x, const void* y)
{
    const ld_arc* a = (const ld_arc*)x;
    const ld_arc* b = (const ld_arc*)y;
    if (a->lab != b->lab) return a->lab < b->lab ? -1 : 1;
    return a->pos < b->pos ? -1 : (a->pos > b->pos ? 1 : 0);
}

/*
 * Exact coarsest stable refinement with double weights, the lumping of
 * Valmari's minimiser built with MDP_weight_is_double
 * (src/part_ref/MDPmin.cc:107-113, MDP_minimize.cc:567-637): the weight of a
 * node into a block is the double sum of its arcs' weights into that block,
 * rounded to float (MDP_round_weight), and a sum that rounds to zero counts
 * as no arc into the block (MDP_minimize.cc:596-599).  Two nodes are
 * equivalent iff they are in the same block and their rounded sums into
 * every block are equal.  The double sum of a (node, block) pair is taken in
 * arc order (the minimiser adds in the order of its block's members, which
 * gives the same float except when the two double sums fall on different
 * sides of a float rounding boundary).
 *   wt[m] (finite doubles) replaces orc_refine_exact's integer weights; the
 *   other arguments and the result are orc_refine_exact's.
 */
int orc_refine_f64(uint32_t n, const uint64_t* off, const uint32_t* idx, const double* wt,
                   const uint32_t* init, uint32_t* labels_out, uint32_t* rounds_out,
                   uint32_t* blocks_out, uint32_t* round_blocks, uint32_t max_rounds)
{
    *rounds_out = 0; *blocks_out = 0;
    if (n == 0) { if (round_blocks) round_blocks[0] = 0; return 0; }
    uint64_t m = off[n];
    uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* nxt = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* ord = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint64_t* sstart = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint32_t* slen = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* slab = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
    uint64_t* sbits = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
    ld_arc* row = (ld_arc*)malloc(sizeof(ld_arc) * (m ? m : 1));

    uint32_t prev;
    if (init) prev = orc_canonicalize(n, init, cur);
    else { for (uint32_t i = 0; i < n; ++i) cur[i] = 0; prev = 1; }
    if (round_blocks) round_blocks[0] = prev;

    int status = -1;
    uint32_t r = 0;
    while (r < max_rounds) {
        for (uint32_t u = 0; u < n; ++u) {
            uint64_t b = off[u], e = off[u + 1], d = e - b;
            for (uint64_t k = 0; k < d; ++k) {
                row[k].lab = cur[idx[b + k]];
                row[k].pos = (uint32_t)k;
                row[k].w = wt[b + k];
            }
            qsort(row, (size_t)d, sizeof(ld_arc), cmp_ld);
            uint32_t len = 0;
            sstart[u] = b;
            for (uint64_t k = 0; k < d;) {
                uint32_t lab = row[k].lab;
                double s = 0.0;
                while (k < d && row[k].lab == lab) { s += row[k].w; ++k; }
                const float f = (float)s;
                if (f != 0.0f) {
                    uint32_t bits;
                    memcpy(&bits, &f, sizeof bits);
                    slab[b + len] = lab; sbits[b + len] = bits; ++len;
                }
            }
            slen[u] = len;
        }
        exact_ctx c = { cur, sstart, slen, slab, sbits };
        for (uint32_t i = 0; i < n; ++i) ord[i] = i;
        msort_idx(ord, tmp, n, cmp_exact, &c);
        uint32_t blocks = 0, rep = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (i == 0 || cmp_exact(ord[i - 1], ord[i], &c) != 0) { rep = ord[i]; ++blocks; }
            nxt[ord[i]] = rep;
        }
        ++r;
        if (round_blocks) round_blocks[r] = blocks;
        uint32_t* sw = cur; cur = nxt; nxt = sw;
        if (blocks == prev) { status = 0; break; }
        prev = blocks;
    }
    *rounds_out = r;
    *blocks_out = orc_canonicalize(n, cur, labels_out);
    free(cur); free(nxt); free(ord); free(tmp); free(sstart); free(slen);
    free(slab); free(sbits); free(row);
    return status;
}

/* The decimal reader of src/part_ref/reader.cc:110-147, which turns the MDP
 * text's weights into doubles when the minimiser is built with
 * MDP_weight_is_double: signs, then the integer digits (x10 + d), then each
 * fractional digit d added as d x scale with scale divided by 10 per digit.
 * The double it returns is not always the nearest one to the decimal, so the
 * weights given to the other restatements and to the product come from here.
 * Returns the number of characters consumed (0 = no digit). */
size_t orc_reader_decimal(const char* s, double* out)
{
    size_t i = 0;
    int neg = 0;
    while (s[i] == '+' || s[i] == '-') { if (s[i] == '-') neg = !neg; ++i; }
    double result = 0.0;
    int digits = s[i] >= '0' && s[i] <= '9';
    while (s[i] >= '0' && s[i] <= '9') { result *= 10; result += s[i] - '0'; ++i; }
    if (s[i] == '.') {
        ++i;
        digits |= s[i] >= '0' && s[i] <= '9';
        double scale = 1.0;
        while (s[i] >= '0' && s[i] <= '9') { scale /= 10; result += scale * (s[i] - '0'); ++i; }
    }
    if (!digits) return 0;
    *out = neg ? -result : result;
    return i;
}

/* ------------------------------------------------------------------ */
/* arcs-cuda text writer (feeds the reference programs)                */
/* ------------------------------------------------------------------ */

/* Writes "N\nM\n" + one "u wt v" line per arc (webgraph-rs
 * cli/src/to/arcscuda.rs:61-66).  Returns 0 or -1. */
int orc_write_arcs(const char* path, uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt)
{
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    static char buf[1 << 20];
    setvbuf(f, buf, _IOFBF, sizeof buf);
    fprintf(f, "%u\n%llu\n", n, (unsigned long long)off[n]);
    char line[80];
    for (uint32_t u = 0; u < n; ++u) {
        for (uint64_t k = off[u]; k < off[u + 1]; ++k) {
            /* hand-rolled formatting: fprintf is the bottleneck at 1e8 arcs */
            char* p = line + sizeof line;
            *--p = '\n';
            uint32_t v = idx[k];
            do { *--p = (char)('0' + v % 10); v /= 10; } while (v);
            *--p = ' ';
            uint64_t w = wt ? wt[k] : 1u;
            do { *--p = (char)('0' + w % 10); w /= 10; } while (w);
            *--p = ' ';
            uint32_t s = u;
            do { *--p = (char)('0' + s % 10); s /= 10; } while (s);
            fwrite(p, 1, (size_t)(line + sizeof line - p), f);
        }
    }
    return fclose(f) == 0 ? 0 : -1;
}

/* ------------------------------------------------------------------ */
/* restatement of the reference CPU loop (rsc.cpp)                     */
/* ------------------------------------------------------------------ */

/* rsc.cpp:63-69: bijective 64-bit mixer (SplitMix64 finaliser, then x5,
 * rotate left by 7, x9). */
uint64_t orc_rsc_randomize(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z = (z ^ (z >> 31)) * 5u;
    return ((z << 7) | (z >> 57)) * 9u;
}

typedef struct { const uint64_t* z; const uint64_t* w; } rsc_ctx;

static int cmp_rsc(uint32_t a, uint32_t b, const void* vctx)
{
    const rsc_ctx* c = (const rsc_ctx*)vctx;
    if (c->z[a] != c->z[b]) return c->z[a] < c->z[b] ? -1 : 1;
    if (c->w[a] != c->w[b]) return c->w[a] < c->w[b] ? -1 : 1;
    return 0;
}

/*
 * rsc.cpp:103-144 restated: w = 1 for every node (or the dense rank of the
 * given initial colour), z = 0; each round z[u] = sum over u's arcs of
 * randomize(w[v] + it) * wt (rows without arcs keep z = 0), order the nodes by
 * (z, w), give each distinct pair its dense rank, it += 1; stop when the count
 * is unchanged.  rounds_gpu uses the count of distinct initial colours as the
 * starting count, rounds_cpu uses N as rsc.cpp:108-109 does.
 */
int orc_refine_rsc(uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt,
                   const uint32_t* init, uint32_t* labels_out, uint32_t* rounds_gpu,
                   uint32_t* rounds_cpu, uint32_t* blocks_out, uint32_t max_rounds)
{
    *rounds_gpu = *rounds_cpu = *blocks_out = 0;
    if (n == 0) return 0;
    uint64_t* w = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint64_t* z = (uint64_t*)calloc(n, sizeof(uint64_t));
    uint32_t* ord = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* lab = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t count0 = 1;
    if (init) {
        /* dense rank of the initial colour, in increasing colour order */
        for (uint32_t i = 0; i < n; ++i) ord[i] = i;
        const uint32_t* c = init;
        msort_idx(ord, tmp, n, cmp_lab, &c);
        uint64_t rank = 1;
        for (uint32_t i = 0; i < n; ++i) {
            if (i && init[ord[i]] != init[ord[i - 1]]) ++rank;
            w[ord[i]] = rank;
        }
        count0 = (uint32_t)rank;
    } else {
        for (uint32_t i = 0; i < n; ++i) w[i] = 1;
    }
    uint64_t it = 0;
    uint32_t prev_cpu = n, prev_gpu = count0, count = count0;
    int status = -1;
    int gpu_done = 0;
    while (it < max_rounds) {
        for (uint32_t u = 0; u < n; ++u) {
            if (off[u] == off[u + 1]) continue;     /* z stays as it was */
            uint64_t s = 0;
            for (uint64_t k = off[u]; k < off[u + 1]; ++k)
                s += orc_rsc_randomize(w[idx[k]] + it) * (wt ? wt[k] : 1u);
            z[u] = s;
        }
        for (uint32_t i = 0; i < n; ++i) ord[i] = i;
        rsc_ctx c = { z, w };
        msort_idx(ord, tmp, n, cmp_rsc, &c);
        uint64_t rank = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (i && cmp_rsc(ord[i - 1], ord[i], &c) != 0) ++rank;
            lab[ord[i]] = (uint32_t)rank;
        }
        for (uint32_t i = 0; i < n; ++i) w[i] = lab[i];
        count = (uint32_t)rank + 1;
        ++it;
        if (!gpu_done) {
            if (count == prev_gpu) { *rounds_gpu = (uint32_t)it; gpu_done = 1; }
            prev_gpu = count;
        }
        if (count == prev_cpu) { status = 0; break; }
        prev_cpu = count;
    }
    /* the CPU convention can stop one pass before the GPU one (round 1 already
     * yields N blocks); the partition is then final, so one more pass would
     * confirm it */
    if (!gpu_done) *rounds_gpu = (uint32_t)it + 1;
    *rounds_cpu = (uint32_t)it;
    if (it == 0)  /* no pass ran: the initial colours */
        for (uint32_t u = 0; u < n; ++u) lab[u] = (uint32_t)w[u];
    *blocks_out = orc_canonicalize(n, lab, labels_out);
    free(w); free(z); free(ord); free(tmp); free(lab);
    return status;
}


/* ------------------------------------------------------------------ */
/* rsc.cpp:71-144 restated again, multi-threaded (pthreads), u64        */
/* counters throughout: the same arithmetic and the same dense ranks    */
/* as orc_refine_rsc, for graphs whose arcs do not fit in 32 bits       */
/* (R-MAT-28: 8.5 G arcs) and a single thread would take too long.      */
/*                                                                      */
/* Dense ranks in (z, w) order without one global sort: every node goes */
/* to a bucket by a key that is monotone in (z, w) -- z = 0 by the      */
/* range of w, z != 0 by the top bits of z -- buckets are sorted in     */
/* parallel, and a bucket's ranks start after all earlier buckets'.     */
/* ------------------------------------------------------------------ */
#define ORC_WBUCKETS 1024u
#define ORC_ZBITS 12u
#define ORC_BUCKETS (ORC_WBUCKETS + (1u << ORC_ZBITS))

typedef struct {
    uint32_t n, threads;
    const uint64_t* off;
    const uint32_t* idx;
    const uint64_t* wt;
    uint64_t* w;
    uint64_t* z;
    uint32_t* ord;
    uint32_t* tmp;
    uint32_t* lab;
    uint64_t it, wmax;
    uint64_t* cnt;        /* [threads][ORC_BUCKETS]: counts, then scatter cursors */
    uint64_t* bstart;     /* [ORC_BUCKETS + 1] */
    uint64_t* bdist;      /* [ORC_BUCKETS]: distinct pairs, then the bucket's first rank */
    uint32_t* sig_lo;     /* [threads + 1]: signature ranges with equal arc counts */
    uint32_t next;        /* bucket work counter */
} mt_ctx;

typedef struct {
    mt_ctx* c;
    uint32_t t;
} mt_arg;

static uint32_t mt_bucket(const mt_ctx* c, uint32_t u)
{
    if (c->z[u] == 0) return (uint32_t)((c->w[u] * (uint64_t)ORC_WBUCKETS) / (c->wmax + 1u));
    return ORC_WBUCKETS + (uint32_t)(c->z[u] >> (64u - ORC_ZBITS));
}

static void mt_range(const mt_ctx* c, uint32_t t, uint32_t* lo, uint32_t* hi)
{
    *lo = (uint32_t)((uint64_t)c->n * t / c->threads);
    *hi = (uint32_t)((uint64_t)c->n * (t + 1) / c->threads);
}

static void* mt_signatures(void* p)
{
    const mt_arg* a = (const mt_arg*)p;
    const mt_ctx* c = a->c;
    for (uint32_t u = c->sig_lo[a->t]; u < c->sig_lo[a->t + 1]; ++u) {
        if (c->off[u] == c->off[u + 1]) continue; /* z stays as it was */
        uint64_t s = 0;
        for (uint64_t k = c->off[u]; k < c->off[u + 1]; ++k)
            s += orc_rsc_randomize(c->w[c->idx[k]] + c->it) * (c->wt ? c->wt[k] : 1u);
        c->z[u] = s;
    }
    return NULL;
}

static void* mt_count(void* p)
{
    const mt_arg* a = (const mt_arg*)p;
    const mt_ctx* c = a->c;
    uint64_t* cnt = c->cnt + (size_t)a->t * ORC_BUCKETS;
    uint32_t lo, hi;
    mt_range(c, a->t, &lo, &hi);
    memset(cnt, 0, sizeof(uint64_t) * ORC_BUCKETS);
    for (uint32_t u = lo; u < hi; ++u) ++cnt[mt_bucket(c, u)];
    return NULL;
}

static void* mt_scatter(void* p)
{
    const mt_arg* a = (const mt_arg*)p;
    const mt_ctx* c = a->c;
    uint64_t* cur = c->cnt + (size_t)a->t * ORC_BUCKETS;
    uint32_t lo, hi;
    mt_range(c, a->t, &lo, &hi);
    for (uint32_t u = lo; u < hi; ++u) c->ord[cur[mt_bucket(c, u)]++] = u;
    return NULL;
}

static void* mt_sort_buckets(void* p)
{
    mt_ctx* c = ((const mt_arg*)p)->c;
    const rsc_ctx rc = { c->z, c->w };
    for (;;) {
        const uint32_t b = __atomic_fetch_add(&c->next, 1u, __ATOMIC_RELAXED);
        if (b >= ORC_BUCKETS) break;
        const uint64_t s = c->bstart[b], e = c->bstart[b + 1];
        if (s == e) {
            c->bdist[b] = 0;
            continue;
        }
        msort_idx(c->ord + s, c->tmp + s, (size_t)(e - s), cmp_rsc, &rc);
        uint64_t r = 0;
        for (uint64_t i = s; i < e; ++i) {
            if (i > s && cmp_rsc(c->ord[i - 1], c->ord[i], &rc) != 0) ++r;
            c->lab[c->ord[i]] = (uint32_t)r;
        }
        c->bdist[b] = r + 1;
    }
    return NULL;
}

static void* mt_apply(void* p)
{
    mt_ctx* c = ((const mt_arg*)p)->c;
    for (;;) {
        const uint32_t b = __atomic_fetch_add(&c->next, 1u, __ATOMIC_RELAXED);
        if (b >= ORC_BUCKETS) break;
        for (uint64_t i = c->bstart[b]; i < c->bstart[b + 1]; ++i) {
            const uint32_t v = c->ord[i];
            c->lab[v] += (uint32_t)c->bdist[b];
            c->w[v] = c->lab[v];
        }
    }
    return NULL;
}

/* Runs fn for every thread index; a thread that cannot be created runs
 * inline. */
static void mt_run(mt_ctx* c, void* (*fn)(void*))
{
    pthread_t th[256];
    mt_arg args[256];
    int made[256];
    for (uint32_t t = 0; t < c->threads; ++t) {
        args[t].c = c;
        args[t].t = t;
        made[t] = pthread_create(&th[t], NULL, fn, &args[t]) == 0;
        if (!made[t]) fn(&args[t]);
    }
    for (uint32_t t = 0; t < c->threads; ++t)
        if (made[t]) pthread_join(th[t], NULL);
}

/* Same contract and results as orc_refine_rsc (labels, rounds in both
 * conventions, blocks); threads in 1..256.  Returns -1 when max_rounds ran
 * out, -2 when memory is short. */
int orc_refine_rsc_mt(uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt,
                      const uint32_t* init, uint32_t* labels_out, uint32_t* rounds_gpu,
                      uint32_t* rounds_cpu, uint32_t* blocks_out, uint32_t max_rounds, uint32_t threads)
{
    *rounds_gpu = *rounds_cpu = *blocks_out = 0;
    if (n == 0) return 0;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    mt_ctx c;
    memset(&c, 0, sizeof c);
    c.n = n;
    c.threads = threads;
    c.off = off;
    c.idx = idx;
    c.wt = wt;
    c.w = (uint64_t*)malloc(sizeof(uint64_t) * n);
    c.z = (uint64_t*)calloc(n, sizeof(uint64_t));
    c.ord = (uint32_t*)malloc(sizeof(uint32_t) * n);
    c.tmp = (uint32_t*)malloc(sizeof(uint32_t) * n);
    c.lab = (uint32_t*)malloc(sizeof(uint32_t) * n);
    c.cnt = (uint64_t*)malloc(sizeof(uint64_t) * ORC_BUCKETS * threads);
    c.bstart = (uint64_t*)malloc(sizeof(uint64_t) * (ORC_BUCKETS + 1));
    c.bdist = (uint64_t*)malloc(sizeof(uint64_t) * ORC_BUCKETS);
    c.sig_lo = (uint32_t*)malloc(sizeof(uint32_t) * (threads + 1));
    int status = -1;
    if (!c.w || !c.z || !c.ord || !c.tmp || !c.lab || !c.cnt || !c.bstart || !c.bdist || !c.sig_lo) {
        status = -2;
        goto out;
    }
    /* signature ranges: equal shares of the arcs (first node whose offset
     * reaches t * m / threads) */
    {
        const uint64_t m = off[n];
        uint32_t u = 0;
        for (uint32_t t = 0; t <= threads; ++t) {
            const uint64_t target = t == threads ? m + 1 : m / threads * t;
            while (u < n && off[u] < target) ++u;
            c.sig_lo[t] = t == threads ? n : u;
        }
        c.sig_lo[0] = 0;
    }
    uint32_t count0 = 1;
    if (init) {
        /* dense rank of the initial colour, in increasing colour order */
        for (uint32_t i = 0; i < n; ++i) c.ord[i] = i;
        const uint32_t* ic = init;
        msort_idx(c.ord, c.tmp, n, cmp_lab, &ic);
        uint64_t rank = 1;
        for (uint32_t i = 0; i < n; ++i) {
            if (i && init[c.ord[i]] != init[c.ord[i - 1]]) ++rank;
            c.w[c.ord[i]] = rank;
        }
        count0 = (uint32_t)rank;
        c.wmax = rank;
    } else {
        for (uint32_t i = 0; i < n; ++i) c.w[i] = 1;
        c.wmax = 1;
    }
    uint32_t prev_cpu = n, prev_gpu = count0, count = count0;
    int gpu_done = 0;
    while (c.it < max_rounds) {
        mt_run(&c, mt_signatures);
        mt_run(&c, mt_count);
        uint64_t pos = 0;
        for (uint32_t b = 0; b < ORC_BUCKETS; ++b) {
            c.bstart[b] = pos;
            for (uint32_t t = 0; t < threads; ++t) {
                const uint64_t k = c.cnt[(size_t)t * ORC_BUCKETS + b];
                c.cnt[(size_t)t * ORC_BUCKETS + b] = pos;
                pos += k;
            }
        }
        c.bstart[ORC_BUCKETS] = pos;
        mt_run(&c, mt_scatter);
        c.next = 0;
        mt_run(&c, mt_sort_buckets);
        uint64_t total = 0;
        for (uint32_t b = 0; b < ORC_BUCKETS; ++b) {
            const uint64_t d = c.bdist[b];
            c.bdist[b] = total;
            total += d;
        }
        c.next = 0;
        mt_run(&c, mt_apply);
        count = (uint32_t)total;
        c.wmax = total ? total - 1 : 0;
        ++c.it;
        if (!gpu_done) {
            if (count == prev_gpu) { *rounds_gpu = (uint32_t)c.it; gpu_done = 1; }
            prev_gpu = count;
        }
        if (count == prev_cpu) { status = 0; break; }
        prev_cpu = count;
    }
    if (!gpu_done) *rounds_gpu = (uint32_t)c.it + 1;
    *rounds_cpu = (uint32_t)c.it;
    /* the ranks are dense (0..count-1): canonical label = first node of
     * each rank, in one pass (c.tmp holds first[rank]) */
    if (c.it == 0) {  /* no pass ran: the initial colours */
        for (uint32_t u = 0; u < n; ++u) c.lab[u] = (uint32_t)c.w[u];
        *blocks_out = orc_canonicalize(n, c.lab, labels_out);
    } else {
        for (uint32_t r = 0; r < count; ++r) c.tmp[r] = UINT32_MAX;
        for (uint32_t u = 0; u < n; ++u) {
            const uint32_t r = c.lab[u];
            if (c.tmp[r] == UINT32_MAX) c.tmp[r] = u;
            labels_out[u] = c.tmp[r];
        }
        *blocks_out = count;
    }
out:
    free(c.w); free(c.z); free(c.ord); free(c.tmp); free(c.lab);
    free(c.cnt); free(c.bstart); free(c.bdist); free(c.sig_lo);
    return status;
}

/* batches = ceil((double)edge_n / max_batch_edge_n) (rbsc.cu:295) */
static double ceil_u64_div_double(uint64_t a, uint64_t b)
{
    const double q = (double)a / (double)b;
    const double t = (double)(uint64_t)q;
    return t < q ? t + 1.0 : t;
}

/* ceil(new_edge_n / (float)max_batch_edge_n) in single precision
 * (rbsc_aggressive.cu:487) */
static float ceilf_u64_div_float(uint64_t a, uint64_t b)
{
    const float q = (float)a / (float)b;
    const float t = (float)(uint64_t)q;
    return t < q ? t + 1.0f : t;
}

/* ------------------------------------------------------------------ */
/* the reference GPU program's edge-batch (quotient) mode              */
/* ------------------------------------------------------------------ */
#define ORC_OFF_BATCH 0
#define ORC_IN_BATCH 1
#define ORC_DANGLING 2
#define ORC_NOT_INIT UINT64_MAX

/*
 * The outer loop of src/rbsc/rbsc.cu:292-487 for one GPU, restated; the stop
 * test of src/rbsc/rbsc_aggressive.cu:487 when `aggressive` is set.  Each
 * batch's local refinement (rbsc.cu:346-425: in-batch sources start in one
 * block, dangling nodes of batch 0 in another, every other node alone;
 * refined over the batch's arcs to the fixpoint) is computed exactly by
 * orc_refine_exact instead of by hashed sums.
 *
 *   off/idx/wt: the graph; its rows in node order are the reference's arc
 *     list grouped by start (rbsc.cu:168-180).
 *   batch: max_batch_edge_n (rbsc.cu:204); 0 = all arcs.
 *   labels_out[n]: canonical labels of the final partition: each original
 *     node's class after the last iteration, composed over the iterations.
 *   blocks_out: new_node_n, the "nodes" line (rbsc.cu:494); done_out: 1 iff
 *     the last iteration had one batch (rbsc.cu:493); iters_out: iterations.
 * Returns 0.  A graph without arcs has no batch: blocks 0, done 0, as the
 * reference prints; its labels are then the coarsest partition (one block).
 */
int orc_refine_edge_batches(uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt, uint64_t batch,
                            int aggressive, uint32_t* labels_out, uint32_t* blocks_out, uint32_t* done_out,
                            uint32_t* iters_out)
{
    const uint64_t E = off[n];
    uint32_t* es = (uint32_t*)malloc(sizeof(uint32_t) * (E ? E : 1));
    uint32_t* ee = (uint32_t*)malloc(sizeof(uint32_t) * (E ? E : 1));
    uint64_t* ew = (uint64_t*)malloc(sizeof(uint64_t) * (E ? E : 1));
    for (uint32_t u = 0; u < n; ++u)
        for (uint64_t k = off[u]; k < off[u + 1]; ++k) {
            es[k] = u;
            ee[k] = idx[k];
            ew[k] = wt ? wt[k] : 1u;
        }
    size_t nn = n ? n : 1;
    uint32_t* cls = (uint32_t*)malloc(sizeof(uint32_t) * nn);
    uint32_t* w = (uint32_t*)malloc(sizeof(uint32_t) * nn);
    uint8_t* mask = (uint8_t*)malloc(nn);
    uint32_t* lab = (uint32_t*)malloc(sizeof(uint32_t) * nn);
    uint32_t* init = (uint32_t*)malloc(sizeof(uint32_t) * nn);
    uint32_t* label_map = (uint32_t*)malloc(sizeof(uint32_t) * nn);
    uint64_t* loff = (uint64_t*)malloc(sizeof(uint64_t) * (nn + 1));
    uint32_t* lidx = (uint32_t*)malloc(sizeof(uint32_t) * (E ? E : 1));
    uint64_t* lwt = (uint64_t*)malloc(sizeof(uint64_t) * (E ? E : 1));
    uint64_t* widx = (uint64_t*)malloc(sizeof(uint64_t) * nn);
    uint8_t* considered = (uint8_t*)malloc(nn);
    for (uint32_t u = 0; u < n; ++u) cls[u] = u;
    if (batch == 0) batch = E ? E : 1;

    uint32_t node_n = n, new_node_n = n, iters = 0;
    uint64_t edge_n = E, new_edge_n = E, batches = 0;
    do {
        node_n = new_node_n;
        edge_n = new_edge_n;
        new_node_n = 0;
        batches = (uint64_t)ceil_u64_div_double(edge_n, batch);
        for (uint32_t i = 0; i < node_n; ++i) w[i] = node_n;
        for (uint64_t b = 0; b < batches; ++b) {
            uint64_t bs = b * batch, be = bs + batch < edge_n ? bs + batch : edge_n;
            for (uint32_t i = 0; i < node_n; ++i) mask[i] = b == 0 ? ORC_DANGLING : ORC_OFF_BATCH;
            uint64_t nbs = ORC_NOT_INIT, nbe = ORC_NOT_INIT;
            for (uint64_t i = bs; i < be; ++i) {
                if ((!i || es[i - 1] != es[i]) && nbs == ORC_NOT_INIT) nbs = i;
                if (i && nbs != ORC_NOT_INIT && es[i - 1] != es[i]) nbe = i;
                mask[es[i]] = ORC_IN_BATCH;
            }
            if (be == edge_n || es[be] != es[be - 1]) nbe = be;
            if (nbs == ORC_NOT_INIT || nbe == ORC_NOT_INIT) continue;
            for (uint64_t i = 0; i < nbs; ++i) mask[es[i]] = ORC_OFF_BATCH;
            for (uint64_t i = nbe; i < edge_n; ++i) mask[es[i]] = ORC_OFF_BATCH;
            /* the batch as a CSR over all node_n nodes (rows in node order) */
            for (uint32_t i = 0; i <= node_n; ++i) loff[i] = 0;
            for (uint64_t i = nbs; i < nbe; ++i) ++loff[es[i] + 1];
            for (uint32_t i = 0; i < node_n; ++i) loff[i + 1] += loff[i];
            for (uint32_t i = 0; i < node_n; ++i) widx[i] = loff[i];
            for (uint64_t i = nbs; i < nbe; ++i) {
                const uint64_t p = widx[es[i]]++;
                lidx[p] = ee[i];
                lwt[p] = ew[i];
            }
            for (uint32_t i = 0; i < node_n; ++i)
                init[i] = mask[i] == ORC_IN_BATCH ? 0u : (mask[i] == ORC_DANGLING ? 1u : i + 2u);
            uint32_t r = 0, bl = 0;
            orc_refine_exact(node_n, loff, lidx, lwt, init, lab, &r, &bl, NULL, node_n + 2);
            /* fresh global ids in the order the batch's classes first appear (rbsc.cu:427-445) */
            for (uint32_t i = 0; i < node_n; ++i) label_map[i] = node_n;
            for (uint32_t i = 0; i < node_n; ++i) {
                if (!mask[i]) continue;
                const uint32_t l = lab[i];
                if (label_map[l] == node_n) label_map[l] = new_node_n++;
                w[i] = label_map[l];
            }
        }
        if (batches > 1) {
            /* quotient (rbsc.cu:451-487): one representative run per class,
             * heads renamed to classes, parallel arcs merged, arc order kept */
            new_edge_n = 0;
            uint64_t first_edge_i = 0;
            uint32_t current_node = 0;
            int counting = 0;
            for (uint32_t i = 0; i < node_n; ++i) {
                widx[i] = edge_n;
                considered[i] = 0;
                if (w[i] == node_n) w[i] = new_node_n++;
            }
            for (uint64_t i = 0; i < edge_n; ++i) {
                if (!i || es[i] != current_node) {
                    current_node = es[i];
                    counting = !considered[w[current_node]];
                    first_edge_i = new_edge_n;
                    considered[w[es[i]]] = 1;
                }
                if (counting) {
                    es[i] = w[es[i]];
                    ee[i] = w[ee[i]];
                    if (widx[ee[i]] == edge_n || widx[ee[i]] < first_edge_i) {
                        es[new_edge_n] = es[i];
                        ee[new_edge_n] = ee[i];
                        ew[new_edge_n] = ew[i];
                        widx[ee[i]] = new_edge_n;
                        ++new_edge_n;
                    } else {
                        ew[widx[ee[i]]] += ew[i];
                    }
                }
            }
        }
        if (batches > 0)
            for (uint32_t u = 0; u < n; ++u) cls[u] = w[cls[u]];
        ++iters;
    } while (batches > 1 && node_n > new_node_n &&
             (!aggressive || (float)batches > ceilf_u64_div_float(new_edge_n, batch)));

    if (batches == 0) for (uint32_t u = 0; u < n; ++u) cls[u] = 0;
    orc_canonicalize(n, cls, labels_out);
    *blocks_out = new_node_n;
    *done_out = batches == 1;
    *iters_out = iters;
    free(es); free(ee); free(ew); free(cls); free(w); free(mask); free(lab); free(init); free(label_map);
    free(loff); free(lidx); free(lwt); free(widx); free(considered);
    return 0;
}

/* ------------------------------------------------------------------ */
/* workload generator and reference-format writers                     */
/* ------------------------------------------------------------------ */
/*
 * The checkers and the CPU baseline build their inputs here, so that nothing
 * that times or checks the product has to load the product library.
 *
 * R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004) with counter-based draws:
 * arc e of m0 = edge_factor * 2^scale starts from base = fmix64(seed ^ e *
 * 0x9E3779B97F4A7C15); at level l = 0 .. scale-1 the draw r is the high 32
 * bits of fmix64(base + (l + 1) * 0xD1B54A32D192ED03), and the quadrant bits
 * are u_bit = (r >= T_ab), v_bit = (T_a <= r < T_ab) or (r >= T_abc), with
 * T_x = floor(x * 2^32) (0xFFFFFFFF at the top).  Duplicate arcs and
 * self-loops are dropped and every row is sorted by head.  These are the
 * rules of the product's generator (gen.cu), restated, so the two produce the
 * same graph; tests compare them.
 */
static uint64_t orc_fmix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

static uint32_t orc_thr(double x)
{
    if (x <= 0) return 0;
    const double t = x * 4294967296.0;
    return t >= 4294967295.0 ? 0xffffffffu : (uint32_t)t;
}

typedef struct {
    uint64_t seed, m0;
    uint32_t scale, ta, tab, tabc, threads;
    uint64_t* cur;      /* [n]: row counts, then scatter cursors */
    uint32_t* heads;    /* [m0]: raw heads by row */
    const uint64_t* raw;/* [n + 1]: raw row offsets */
    uint64_t* keep;     /* [n]: heads kept per row */
    uint64_t* off;      /* [n + 1] final */
    uint32_t* idx;      /* final heads */
    uint64_t next;      /* row-chunk work counter */
    int phase;
} gen_ctx;

static void orc_rmat_arc(const gen_ctx* g, uint64_t e, uint32_t* u, uint32_t* v)
{
    const uint64_t base = orc_fmix64(g->seed ^ (e * 0x9E3779B97F4A7C15ULL));
    uint32_t uu = 0, vv = 0;
    for (uint32_t l = 0; l < g->scale; ++l) {
        const uint32_t r = (uint32_t)(orc_fmix64(base + (uint64_t)(l + 1) * 0xd1b54a32d192ed03ULL) >> 32);
        uu = (uu << 1) | (r >= g->tab ? 1u : 0u);
        vv = (vv << 1) | (((r >= g->ta && r < g->tab) || r >= g->tabc) ? 1u : 0u);
    }
    *u = uu;
    *v = vv;
}

static int cmp_u32(const void* x, const void* y)
{
    const uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
    return a < b ? -1 : a > b;
}

#define GEN_ROW_CHUNK 4096u

typedef struct { gen_ctx* g; uint32_t t; } gen_arg;

static void* gen_worker(void* p)
{
    const gen_arg* a = (const gen_arg*)p;
    gen_ctx* g = a->g;
    const uint64_t n = 1ull << g->scale;
    if (g->phase == 0 || g->phase == 1) {  /* count, then scatter, over this thread's arcs */
        const uint64_t lo = g->m0 * a->t / g->threads, hi = g->m0 * (a->t + 1) / g->threads;
        for (uint64_t e = lo; e < hi; ++e) {
            uint32_t u, v;
            orc_rmat_arc(g, e, &u, &v);
            const uint64_t pos = __atomic_fetch_add(&g->cur[u], 1ull, __ATOMIC_RELAXED);
            if (g->phase == 1) g->heads[pos] = v;
        }
        return NULL;
    }
    for (;;) {  /* rows in chunks: sort + dedup (phase 2), copy (phase 3) */
        const uint64_t c0 = __atomic_fetch_add(&g->next, (uint64_t)GEN_ROW_CHUNK, __ATOMIC_RELAXED);
        if (c0 >= n) break;
        const uint64_t c1 = c0 + GEN_ROW_CHUNK < n ? c0 + GEN_ROW_CHUNK : n;
        for (uint64_t u = c0; u < c1; ++u) {
            uint32_t* r = g->heads + g->raw[u];
            const uint64_t len = g->raw[u + 1] - g->raw[u];
            if (g->phase == 2) {
                if (len <= 32) {
                    for (uint64_t i = 1; i < len; ++i) {
                        const uint32_t x = r[i];
                        uint64_t j = i;
                        while (j > 0 && r[j - 1] > x) { r[j] = r[j - 1]; --j; }
                        r[j] = x;
                    }
                } else {
                    qsort(r, (size_t)len, sizeof(uint32_t), cmp_u32);
                }
                uint64_t k = 0;
                for (uint64_t i = 0; i < len; ++i)
                    if ((i == 0 || r[i] != r[i - 1]) && r[i] != (uint32_t)u) r[k++] = r[i];
                g->keep[u] = k;
            } else {
                memcpy(g->idx + g->off[u], r, sizeof(uint32_t) * g->keep[u]);
            }
        }
    }
    return NULL;
}

static void gen_run(gen_ctx* g, int phase)
{
    pthread_t th[256];
    gen_arg args[256];
    int made[256];
    g->phase = phase;
    g->next = 0;
    for (uint32_t t = 0; t < g->threads; ++t) {
        args[t].g = g;
        args[t].t = t;
        made[t] = pthread_create(&th[t], NULL, gen_worker, &args[t]) == 0;
        if (!made[t]) gen_worker(&args[t]);
    }
    for (uint32_t t = 0; t < g->threads; ++t)
        if (made[t]) pthread_join(th[t], NULL);
}

/* R-MAT graph as CSR (malloc'd; release with orc_free).  Returns 0, -1 for
 * bad sizes, -2 when memory is short. */
int orc_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, uint32_t threads,
                 uint64_t** off_out, uint32_t** idx_out, uint64_t* m_out)
{
    *off_out = NULL;
    *idx_out = NULL;
    *m_out = 0;
    if (scale < 1 || scale > 30 || edge_factor == 0) return -1;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    const uint64_t n = 1ull << scale;
    gen_ctx g;
    memset(&g, 0, sizeof g);
    g.seed = seed;
    g.scale = scale;
    g.m0 = (uint64_t)edge_factor << scale;
    g.ta = orc_thr(a);
    g.tab = orc_thr(a + b);
    g.tabc = orc_thr(a + b + c);
    g.threads = threads;
    uint64_t* raw = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    g.cur = (uint64_t*)calloc(n, sizeof(uint64_t));
    g.heads = (uint32_t*)malloc(sizeof(uint32_t) * g.m0);
    g.keep = (uint64_t*)malloc(sizeof(uint64_t) * n);
    g.off = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    if (!raw || !g.cur || !g.heads || !g.keep || !g.off) {
        free(raw); free(g.cur); free(g.heads); free(g.keep); free(g.off);
        return -2;
    }
    gen_run(&g, 0);
    raw[0] = 0;
    for (uint64_t u = 0; u < n; ++u) {
        raw[u + 1] = raw[u] + g.cur[u];
        g.cur[u] = raw[u];
    }
    g.raw = raw;
    gen_run(&g, 1);
    gen_run(&g, 2);
    g.off[0] = 0;
    for (uint64_t u = 0; u < n; ++u) g.off[u + 1] = g.off[u] + g.keep[u];
    g.idx = (uint32_t*)malloc(sizeof(uint32_t) * (g.off[n] ? g.off[n] : 1));
    if (!g.idx) {
        free(raw); free(g.cur); free(g.heads); free(g.keep); free(g.off);
        return -2;
    }
    gen_run(&g, 3);
    free(raw); free(g.cur); free(g.heads); free(g.keep);
    *off_out = g.off;
    *idx_out = g.idx;
    *m_out = g.off[n];
    return 0;
}

void orc_free(void* p) { free(p); }

static char* put_u64(char* end, uint64_t x)
{
    do { *--end = (char)('0' + x % 10); x /= 10; } while (x);
    return end;
}

/* Valmari MDP text (src/part_ref/MDP_read.cc:51-63, as valmari-adapter:9-16
 * converts arcs-cuda): "n 0 0 m nb", then one "u+1 w v+1" line per arc, then
 * for every initial colour but the smallest its member states (1-based,
 * increasing) followed by 0 -- block 1 is the rest (MDP_read.cc:140-150).
 * init NULL = one block.  Returns 0 or -1. */
int orc_write_mdp(const char* path, uint32_t n, const uint64_t* off, const uint32_t* idx, const uint64_t* wt,
                  const uint32_t* init)
{
    uint32_t* colours = NULL;
    uint32_t* order = NULL;
    uint64_t* start = NULL;
    uint32_t nc = 1;
    if (init && n) {
        colours = (uint32_t*)malloc(sizeof(uint32_t) * n);
        if (!colours) return -1;
        memcpy(colours, init, sizeof(uint32_t) * n);
        qsort(colours, n, sizeof(uint32_t), cmp_u32);
        nc = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (i == 0 || colours[i] != colours[i - 1]) colours[nc++] = colours[i];
        /* members per colour rank, by counting sort (increasing node id) */
        start = (uint64_t*)calloc((size_t)nc + 1, sizeof(uint64_t));
        order = (uint32_t*)malloc(sizeof(uint32_t) * n);
        uint32_t* rank = (uint32_t*)malloc(sizeof(uint32_t) * n);
        if (!start || !order || !rank) { free(colours); free(start); free(order); free(rank); return -1; }
        for (uint32_t u = 0; u < n; ++u) {
            uint32_t lo = 0, hi = nc;
            while (hi - lo > 1) { const uint32_t mid = (lo + hi) / 2; if (colours[mid] <= init[u]) lo = mid; else hi = mid; }
            rank[u] = lo;
            ++start[lo + 1];
        }
        for (uint32_t r = 0; r < nc; ++r) start[r + 1] += start[r];
        uint64_t* pos = (uint64_t*)malloc(sizeof(uint64_t) * nc);
        if (!pos) { free(colours); free(start); free(order); free(rank); return -1; }
        memcpy(pos, start, sizeof(uint64_t) * nc);
        for (uint32_t u = 0; u < n; ++u) order[pos[rank[u]]++] = u;
        free(pos);
        free(rank);
    }
    FILE* f = fopen(path, "w");
    if (!f) { free(colours); free(start); free(order); return -1; }
    static char buf[1 << 20];
    setvbuf(f, buf, _IOFBF, sizeof buf);
    fprintf(f, "%u 0 0 %llu %u\n", n, (unsigned long long)(n ? off[n] : 0), nc);
    char line[80];
    for (uint32_t u = 0; u < n; ++u)
        for (uint64_t k = off[u]; k < off[u + 1]; ++k) {
            char* p = line + sizeof line;
            *--p = '\n';
            p = put_u64(p, (uint64_t)idx[k] + 1u);
            *--p = ' ';
            p = put_u64(p, wt ? wt[k] : 1u);
            *--p = ' ';
            p = put_u64(p, (uint64_t)u + 1u);
            fwrite(p, 1, (size_t)(line + sizeof line - p), f);
        }
    for (uint32_t r = 1; init && r < nc; ++r) {
        for (uint64_t i = start[r]; i < start[r + 1]; ++i) {
            char* p = line + sizeof line;
            *--p = ' ';
            p = put_u64(p, (uint64_t)order[i] + 1u);
            fwrite(p, 1, (size_t)(line + sizeof line - p), f);
        }
        fputs("0\n", f);
    }
    free(colours); free(start); free(order);
    return fclose(f) == 0 ? 0 : -1;
}
