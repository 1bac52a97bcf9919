"""Seeded synthetic graphs (CSR with uint64 offsets and uint32 heads).

These stand in for the reference's LAW web graphs (bench.db), which need the
network and the Rust webgraph decoder.  Row u lists the heads v of the arcs
(u, v): the arcs-cuda convention of the reference (arcs grouped by start).
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def csr_from_arcs(n: int, src, dst, wt=None, sort: bool = True):
    """Arcs -> CSR.  With sort=True rows are sorted by head (stable)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if sort:
        order = np.lexsort((dst, src))
    else:
        order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    w = None if wt is None else np.asarray(wt, dtype=np.uint64)[order]
    off = np.zeros(n + 1, dtype=np.uint64)
    if src.size:
        np.add.at(off, src + 1, 1)
    off = np.cumsum(off, dtype=np.uint64)
    return off, dst.astype(np.uint32), w


def arcs_of(off, idx):
    off = np.asarray(off, dtype=np.int64)
    src = np.repeat(np.arange(len(off) - 1, dtype=np.int64), np.diff(off))
    return src, np.asarray(idx, dtype=np.int64)


def dedup(n, src, dst, drop_self_loops=True):
    key = np.asarray(src, dtype=np.int64) * n + np.asarray(dst, dtype=np.int64)
    key = np.unique(key)
    s, d = key // n, key % n
    if drop_self_loops:
        keep = s != d
        s, d = s[keep], d[keep]
    return s, d


# ---------------------------------------------------------------- workloads

def er_directed(n: int, m: int, seed: int):
    """m distinct directed arcs without self-loops, uniform."""
    rng = np.random.default_rng(seed)
    assert m <= n * (n - 1)
    keys = np.zeros(0, dtype=np.int64)
    while keys.size < m:
        need = m - keys.size
        s = rng.integers(0, n, size=2 * need + 16)
        d = rng.integers(0, n, size=2 * need + 16)
        ok = s != d
        keys = np.unique(np.concatenate([keys, s[ok] * n + d[ok]]))
        if keys.size > m:
            keys = rng.choice(keys, size=m, replace=False)
    return csr_from_arcs(n, keys // n, keys % n)[:2]


def random_lift(base_n: int = 4096, base_m: int = 32768, lift: int = 32, seed: int = 1):
    """Directed random lift: base ER graph, every base node copied `lift`
    times, every base arc (u, v) becomes arcs (u*lift+i, v*lift+pi(i)) for a
    uniform permutation pi per base arc.  Defaults: the 131,072-node /
    1,048,576-arc plain-refinement workload."""
    boff, bidx = er_directed(base_n, base_m, seed)
    bs, bd = arcs_of(boff, bidx)
    rng = np.random.default_rng(seed + 0x51F7)
    perms = np.argsort(rng.random((bs.size, lift)), axis=1)
    i = np.arange(lift, dtype=np.int64)
    src = (bs[:, None] * lift + i[None, :]).ravel()
    dst = (bd[:, None] * lift + perms).ravel()
    return csr_from_arcs(base_n * lift, src, dst)[:2]


def _fmix64(k):
    k = k.astype(np.uint64)
    k ^= k >> np.uint64(33)
    k *= np.uint64(0xFF51AFD7ED558CCD)
    k ^= k >> np.uint64(33)
    k *= np.uint64(0xC4CEB9FE1A85EC53)
    k ^= k >> np.uint64(33)
    return k


def _thr(x: float) -> np.uint64:
    if x <= 0:
        return np.uint64(0)
    t = x * 4294967296.0
    return np.uint64(0xFFFFFFFF if t >= 4294967295.0 else int(t))


def rmat(scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed: int = 1):
    """The counter-based R-MAT of librbsc (gen.cu), in numpy: same arcs as
    rbsc_gen_rmat_host / rbsc_gen_rmat_device.  Duplicates and self-loops
    removed, rows sorted."""
    n = 1 << scale
    m0 = edge_factor << scale
    ta, tab, tabc = _thr(a), _thr(a + b), _thr(a + b + c)
    with np.errstate(over="ignore"):
        e = np.arange(m0, dtype=np.uint64)
        base = _fmix64(np.uint64(seed) ^ (e * GOLDEN))
        u = np.zeros(m0, dtype=np.uint64)
        v = np.zeros(m0, dtype=np.uint64)
        for lvl in range(scale):
            r = _fmix64(base + np.uint64(lvl + 1) * np.uint64(0xD1B54A32D192ED03)) >> np.uint64(32)
            ub = (r >= tab).astype(np.uint64)
            vb = (((r >= ta) & (r < tab)) | (r >= tabc)).astype(np.uint64)
            u = (u << np.uint64(1)) | ub
            v = (v << np.uint64(1)) | vb
    s, d = dedup(n, u.astype(np.int64), v.astype(np.int64))
    return csr_from_arcs(n, s, d)[:2]


def er_undirected(n: int, mean_degree: float, seed: int):
    """Symmetric arcs of an undirected G(n, p), p = mean_degree / (n - 1)."""
    rng = np.random.default_rng(seed)
    if n < 2:
        return csr_from_arcs(n, [], [])[:2]
    p = min(1.0, mean_degree / (n - 1))
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.size) < p
    s, d = iu[keep], ju[keep]
    return csr_from_arcs(n, np.concatenate([s, d]), np.concatenate([d, s]))[:2]


def random_regular(n: int, d: int, seed: int, tries: int = 1000):
    """Symmetric arcs of a uniform-ish simple d-regular graph (pairing model
    with restarts).  n*d must be even."""
    assert (n * d) % 2 == 0
    rng = np.random.default_rng(seed)
    for _ in range(tries):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        if np.unique(lo * n + hi).size != lo.size:
            continue
        return csr_from_arcs(n, np.concatenate([a, b]), np.concatenate([b, a]))[:2]
    raise RuntimeError("random_regular: no simple pairing found")


# ---------------------------------------------------------- known answers

def cycle(n: int):
    return csr_from_arcs(n, np.arange(n), (np.arange(n) + 1) % n)[:2]


def path(n: int):
    return csr_from_arcs(n, np.arange(n - 1), np.arange(1, n))[:2]


def star_out(n: int):
    """Node 0 -> every other node."""
    return csr_from_arcs(n, np.zeros(n - 1, dtype=np.int64), np.arange(1, n))[:2]


def complete_bipartite(a: int, b: int):
    s = np.repeat(np.arange(a), b)
    d = np.tile(np.arange(a, a + b), a)
    return csr_from_arcs(a + b, np.concatenate([s, d]), np.concatenate([d, s]))[:2]


def two_triangles_and_hexagon():
    """Undirected two disjoint triangles (nodes 0-5) plus a 6-cycle (6-11):
    both 2-regular, so 1-WL cannot tell them apart: one block."""
    s, d = [], []
    for t in (0, 3):
        for i in range(3):
            s += [t + i, t + (i + 1) % 3]
            d += [t + (i + 1) % 3, t + i]
    for i in range(6):
        s += [6 + i, 6 + (i + 1) % 6]
        d += [6 + (i + 1) % 6, 6 + i]
    return csr_from_arcs(12, s, d)[:2]


def disjoint_union(graphs):
    """Concatenate CSRs; returns (off, idx, node_offsets)."""
    offs, idxs, base, nbase = [], [], 0, [0]
    arc_base = np.uint64(0)
    for off, idx in graphs:
        off = np.asarray(off, dtype=np.uint64)
        n = len(off) - 1
        offs.append(off[:-1] + arc_base)
        idxs.append(np.asarray(idx, dtype=np.uint32) + np.uint32(base))
        arc_base += off[-1]
        base += n
        nbase.append(base)
    offs.append(np.array([arc_base], dtype=np.uint64))
    return np.concatenate(offs), (np.concatenate(idxs) if idxs else np.zeros(0, np.uint32)), np.array(nbase)


def small_graph_mix(count: int, seed: int, n_lo: int = 10, n_hi: int = 500):
    """The batched-sweep workload: `count` graphs with n ~ U[n_lo, n_hi]; half
    undirected ER with mean degree 4, half random 3-regular (odd n rounded
    down to even); labels U{1..8}.  Returns (graphs, labels)."""
    rng = np.random.default_rng(seed)
    graphs, labels = [], []
    for g in range(count):
        n = int(rng.integers(n_lo, n_hi + 1))
        if g % 2 == 0:
            graphs.append(er_undirected(n, 4.0, int(rng.integers(1 << 62))))
        else:
            n -= n % 2
            graphs.append(random_regular(n, 3, int(rng.integers(1 << 62))))
        labels.append(rng.integers(1, 9, size=len(graphs[-1][0]) - 1).astype(np.uint32))
    return graphs, labels
