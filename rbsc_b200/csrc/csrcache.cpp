// csrcache.cpp -- a binary cache of a host CSR, so that a graph parsed once
// from arcs-cuda text (or decoded from BV files) loads again without the
// parse.  Little-endian layout:
//   bytes 0-7    magic "RBSCCSR1"
//   8-11         version (2; version 1 files are still read)
//   12-15        flags (bit 0: weights present)
//   16-23        n (nodes)        24-31  m (arcs)
//   32-39        checksum of everything after the header
//   40-63        zero
//   then         offsets uint64[n+1], indices uint32[m], weights uint64[m] if flagged
// Checksum, version 2: each array is cut into 1 MiB blocks; a block's digest
// runs four independent 64-bit lanes over its 8-byte words (multiply, rotate,
// multiply), then folds the lanes, the tail bytes and the block length through
// the MurmurHash3 64-bit finaliser; the blocks' digests are folded in order,
// array after array.  The blocks are digested by several threads.  Version 1
// used FNV-1a 64 over every byte, one serial multiply per byte (~0.45 s for
// R-MAT-22's 295 MB against a ~0.1 s read).
// A file whose size, checksum or offsets do not agree is rejected.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/rbsc.h"

rbsc_status rbsc_fail(struct rbsc_ctx* ctx, rbsc_status code, const char* fmt, ...);

namespace {

constexpr char kMagic[8] = {'R', 'B', 'S', 'C', 'C', 'S', 'R', '1'};
constexpr size_t kHeader = 64;

struct Fnv {
    uint64_t h = 0xcbf29ce484222325ull;
    void add(const void* p, size_t n)
    {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 0x100000001b3ull;
        }
    }
};

constexpr uint32_t kVersion = 2;
constexpr size_t kBlock = size_t(1) << 20;

inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

// MurmurHash3's 64-bit finaliser
inline uint64_t fmix64(uint64_t z)
{
    z ^= z >> 33;
    z *= 0xff51afd7ed558ccdull;
    z ^= z >> 33;
    z *= 0xc4ceb9fe1a85ec53ull;
    z ^= z >> 33;
    return z;
}

uint64_t block_digest(const uint8_t* p, size_t n)
{
    constexpr uint64_t K1 = 0x9e3779b97f4a7c15ull, K2 = 0xbf58476d1ce4e5b9ull;
    uint64_t l0 = K1, l1 = K2, l2 = ~K1, l3 = ~K2;
    size_t i = 0;
    for (; i + 32 <= n; i += 32) {
        uint64_t w[4];
        std::memcpy(w, p + i, 32);
        l0 = rotl64(l0 ^ (w[0] * K1), 31) * K2;
        l1 = rotl64(l1 ^ (w[1] * K1), 31) * K2;
        l2 = rotl64(l2 ^ (w[2] * K1), 31) * K2;
        l3 = rotl64(l3 ^ (w[3] * K1), 31) * K2;
    }
    uint64_t t = 0;
    for (; i < n; ++i) t = (t << 8 | t >> 56) ^ p[i];
    return fmix64(l0 ^ rotl64(l1, 16) ^ rotl64(l2, 32) ^ rotl64(l3, 48) ^ fmix64(t ^ (uint64_t)n));
}

// Version-2 checksum of the arrays, in order.
uint64_t checksum2(const void* const* arrays, const size_t* bytes, int count)
{
    std::vector<const uint8_t*> bp;
    std::vector<size_t> bn;
    for (int a = 0; a < count; ++a)
        for (size_t o = 0; o < bytes[a]; o += kBlock) {
            bp.push_back(static_cast<const uint8_t*>(arrays[a]) + o);
            bn.push_back(std::min(kBlock, bytes[a] - o));
        }
    std::vector<uint64_t> d(bp.size());
    const size_t nb = bp.size();
    const int T = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), std::max<size_t>(1, nb / 4));
    auto work = [&](int t) {
        for (size_t b = (size_t)t; b < nb; b += (size_t)T) d[b] = block_digest(bp[b], bn[b]);
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < T; ++t) ts.emplace_back(work, t);
    work(0);
    for (auto& x : ts) x.join();
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t b = 0; b < nb; ++b) h = rotl64((h ^ d[b]) * 0x100000001b3ull, 29);
    return fmix64(h ^ (uint64_t)nb);
}

void put64(uint8_t* p, uint64_t v) { std::memcpy(p, &v, 8); }
void put32(uint8_t* p, uint32_t v) { std::memcpy(p, &v, 4); }
uint64_t get64(const uint8_t* p) { uint64_t v; std::memcpy(&v, p, 8); return v; }
uint32_t get32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; }

}  // namespace

extern "C" rbsc_status rbsc_csr_save(const char* path, const rbsc_csr* g)
{
    if (!path || !g) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null argument");
    if (g->offset_bytes != 8) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "the cache stores 8-byte offsets");
    if (!g->offsets || (g->m && !g->indices)) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null arrays");
    const uint64_t* off = static_cast<const uint64_t*>(g->offsets);
    if (off[0] != 0 || off[g->n] != g->m) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "offsets do not span [0, M]");
    const void* arr[3] = {off, g->indices, g->weights};
    const size_t len[3] = {8 * ((size_t)g->n + 1), g->m ? 4 * (size_t)g->m : 0,
                           (g->weights && g->m) ? 8 * (size_t)g->m : 0};
    uint8_t h[kHeader] = {};
    std::memcpy(h, kMagic, 8);
    put32(h + 8, kVersion);
    put32(h + 12, g->weights ? 1u : 0u);
    put64(h + 16, g->n);
    put64(h + 24, g->m);
    put64(h + 32, checksum2(arr, len, 3));
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "cannot write %s", path);
    bool ok = std::fwrite(h, 1, kHeader, fp) == kHeader;
    ok = ok && std::fwrite(off, 8, (size_t)g->n + 1, fp) == (size_t)g->n + 1;
    if (g->m) ok = ok && std::fwrite(g->indices, 4, g->m, fp) == g->m;
    if (g->weights && g->m) ok = ok && std::fwrite(g->weights, 8, g->m, fp) == g->m;
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "writing %s failed", path);
    return RBSC_OK;
}

extern "C" rbsc_status rbsc_csr_load(const char* path, rbsc_host_graph* out)
{
    if (!path || !out) return rbsc_fail(nullptr, RBSC_ERR_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return rbsc_fail(nullptr, RBSC_ERR_PARSE, "cannot read %s", path);
    uint8_t h[kHeader];
    auto fail = [&](const char* why) {
        std::fclose(fp);
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: %s", path, why);
    };
    if (std::fread(h, 1, kHeader, fp) != kHeader || std::memcmp(h, kMagic, 8) != 0) return fail("not a CSR cache file");
    const uint32_t version = get32(h + 8);
    if (version != 1 && version != kVersion) return fail("unknown version");
    const bool weighted = (get32(h + 12) & 1u) != 0;
    const uint64_t n = get64(h + 16), m = get64(h + 24), sum = get64(h + 32);
    if (n >= 0x80000000ull) return fail("N must be < 2^31");
    std::fseek(fp, 0, SEEK_END);
    const long long size = std::ftell(fp);
    const long long want = (long long)kHeader + 8ll * (long long)(n + 1) + 4ll * (long long)m + (weighted ? 8ll * (long long)m : 0ll);
    if (size != want) return fail("size does not match the header");
    std::fseek(fp, (long)kHeader, SEEK_SET);
    out->n = (uint32_t)n;
    out->m = m;
    out->offsets = (uint64_t*)std::malloc(8 * (size_t)(n + 1));
    out->indices = (uint32_t*)std::malloc(4 * std::max<size_t>((size_t)m, 1));
    out->weights = weighted ? (uint64_t*)std::malloc(8 * std::max<size_t>((size_t)m, 1)) : nullptr;
    if (!out->offsets || !out->indices || (weighted && !out->weights)) return fail("out of host memory");
    bool ok = std::fread(out->offsets, 8, n + 1, fp) == n + 1;
    if (m) ok = ok && std::fread(out->indices, 4, m, fp) == m;
    if (weighted && m) ok = ok && std::fread(out->weights, 8, m, fp) == m;
    if (!ok) return fail("short read");
    std::fclose(fp);
    uint64_t got = 0;
    if (version == 1) {
        Fnv f;
        f.add(out->offsets, 8 * ((size_t)n + 1));
        if (m) f.add(out->indices, 4 * (size_t)m);
        if (weighted && m) f.add(out->weights, 8 * (size_t)m);
        got = f.h;
    } else {
        const void* arr[3] = {out->offsets, out->indices, out->weights};
        const size_t len[3] = {8 * ((size_t)n + 1), m ? 4 * (size_t)m : 0, (weighted && m) ? 8 * (size_t)m : 0};
        got = checksum2(arr, len, 3);
    }
    auto reject = [&](const char* why) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: %s", path, why);
    };
    if (got != sum) return reject("checksum mismatch");
    if (out->offsets[0] != 0 || out->offsets[n] != m) return reject("offsets do not span [0, M]");
    // offsets non-decreasing and heads < N, checked by several threads
    const int T = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<int> bad(T, 0);
    auto check = [&](int t) {
        const uint64_t* o = out->offsets;
        const uint32_t* ix = out->indices;
        for (uint64_t u = n * t / T; u < n * (t + 1) / T; ++u)
            if (o[u + 1] < o[u]) bad[t] |= 1;
        for (uint64_t k = m * t / T; k < m * (t + 1) / T; ++k)
            if (ix[k] >= n) bad[t] |= 2;
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < T; ++t) ts.emplace_back(check, t);
    check(0);
    for (auto& x : ts) x.join();
    int any = 0;
    for (int b : bad) any |= b;
    if (any & 1) return reject("offsets decrease");
    if (any & 2) return reject("a head is >= N");
    return RBSC_OK;
}
