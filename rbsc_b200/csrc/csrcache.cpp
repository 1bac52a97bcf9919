// csrcache.cpp -- a binary cache of a host CSR, so that a graph parsed once
// from arcs-cuda text (or decoded from BV files) loads again without the
// parse.  Little-endian layout:
//   bytes 0-7    magic "RBSCCSR1"
//   8-11         version (1)      12-15  flags (bit 0: weights present)
//   16-23        n (nodes)        24-31  m (arcs)
//   32-39        FNV-1a 64 checksum of everything after the header
//   40-63        zero
//   then         offsets uint64[n+1], indices uint32[m], weights uint64[m] if flagged
// A file whose size, checksum or offsets do not agree is rejected.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

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
    Fnv f;
    f.add(off, 8 * ((size_t)g->n + 1));
    if (g->m) f.add(g->indices, 4 * (size_t)g->m);
    if (g->weights && g->m) f.add(g->weights, 8 * (size_t)g->m);
    uint8_t h[kHeader] = {};
    std::memcpy(h, kMagic, 8);
    put32(h + 8, 1);
    put32(h + 12, g->weights ? 1u : 0u);
    put64(h + 16, g->n);
    put64(h + 24, g->m);
    put64(h + 32, f.h);
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
    if (get32(h + 8) != 1) return fail("unknown version");
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
    Fnv f;
    f.add(out->offsets, 8 * ((size_t)n + 1));
    if (m) f.add(out->indices, 4 * (size_t)m);
    if (weighted && m) f.add(out->weights, 8 * (size_t)m);
    auto reject = [&](const char* why) {
        rbsc_host_graph_free(out);
        return rbsc_fail(nullptr, RBSC_ERR_PARSE, "%s: %s", path, why);
    };
    if (f.h != sum) return reject("checksum mismatch");
    if (out->offsets[0] != 0 || out->offsets[n] != m) return reject("offsets do not span [0, M]");
    for (uint64_t u = 0; u < n; ++u)
        if (out->offsets[u + 1] < out->offsets[u]) return reject("offsets decrease");
    for (uint64_t k = 0; k < m; ++k)
        if (out->indices[k] >= n) return reject("a head is >= N");
    return RBSC_OK;
}
