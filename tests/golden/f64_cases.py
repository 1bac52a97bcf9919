"""Cases of the double-weight lumping fixtures (tests/golden/f64.json).

Every case is a graph whose arc weights are decimal strings, as the
minimiser's MDP text carries them (src/part_ref/MDP_read.cc:57-61), plus
optional initial colours.  The strings go to the reference minimiser built
with double weights; the doubles its reader makes of them
(src/part_ref/reader.cc:110-147, restated in oracle.c) go to the oracle and to
the product.  Graphs have no parallel arcs (the minimiser's reader takes at
most states-squared transitions, and merging parallel arcs would change the
order of the double sums).
"""
from __future__ import annotations

import numpy as np

POOL = ["0.1", "0.2", "0.3", "0.7", "0.333", "0.667", "-0.5", "0.5", "1.25", "0.001", "12.75", "2", "3", "0.125"]


def _csr(n, rows):
    """rows[u] = [(head, weight text), ...] (heads distinct) -> off, idx, texts."""
    off = np.zeros(n + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    idx = np.array([h for r in rows for h, _ in r], dtype=np.uint32)
    texts = [t for r in rows for _, t in r]
    return off, idx, texts


def known(name):
    """Small cases with a known answer."""
    if name == "float_merge":
        # 0 -> {2: 0.1, 3: 0.2}, 1 -> {4: 0.3}: one block for 0 and 1 (the
        # rounded sums into the sink block agree), one for the sinks
        return _csr(5, [[(2, "0.1"), (3, "0.2")], [(4, "0.3")], [], [], []]), None
    if name == "cancel":
        # 0 -> {2: 0.5, 3: -0.5} sums to zero into the sink block: as no arc
        return _csr(4, [[(2, "0.5"), (3, "-0.5")], [], [], []]), None
    if name == "zero_weight":
        # an arc of weight 0 counts as no arc
        return _csr(4, [[(2, "0")], [(3, "0.0")], [], [(0, "1")]]), None
    if name == "chain_rows_sum_to_one":
        # a Markov chain: two copies of a 3-state chain, one split 0.5 / 0.5
        # over two equivalent targets; lumpable pairwise
        rows = [[(1, "0.25"), (2, "0.75")], [(0, "1")], [(2, "1")],
                [(4, "0.125"), (7, "0.125"), (5, "0.75")], [(3, "1")], [(5, "1")], [(3, "1")], [(3, "1")]]
        return _csr(8, rows), None
    if name == "initial_colours":
        rows = [[(2, "1")], [(3, "1")], [], []]
        return _csr(4, rows), np.array([0, 1, 2, 2], dtype=np.uint32)
    raise KeyError(name)


KNOWN = ["float_merge", "cancel", "zero_weight", "chain_rows_sum_to_one", "initial_colours"]


def lifted(seed: int, base_n: int, lift: int, pool_k: int, colours: int):
    """A random base graph lifted `lift` times: every copy of base node u has
    an arc to one random copy of each of u's base successors, with the base
    arc's weight; the lumping then merges the copies (unless the weights of
    different base arcs collide).  colours > 1: random initial colours per
    base node (shared by its copies)."""
    rng = np.random.default_rng(seed)
    pool = rng.choice(POOL, pool_k, replace=False)
    base = [sorted(set(rng.integers(0, base_n, rng.integers(0, 5)).tolist())) for _ in range(base_n)]
    wt = {(u, v): str(rng.choice(pool)) for u in range(base_n) for v in base[u]}
    rows = []
    for u in range(base_n):
        for _ in range(lift):
            rows.append(sorted((v * lift + int(rng.integers(0, lift)), wt[(u, v)]) for v in base[u]))
    n = base_n * lift
    init = None
    if colours > 1:
        bc = rng.integers(0, colours, base_n)
        init = np.repeat(bc, lift).astype(np.uint32)
    return _csr(n, rows), init


def random_graph(seed: int, n: int, max_deg: int, pool_k: int, colours: int):
    """Random heads (distinct per row), weights from a small pool."""
    rng = np.random.default_rng(seed)
    pool = rng.choice(POOL, pool_k, replace=False)
    rows = []
    for _ in range(n):
        hs = sorted(set(rng.integers(0, n, rng.integers(0, max_deg + 1)).tolist()))
        rows.append([(h, str(rng.choice(pool))) for h in hs])
    init = rng.integers(0, colours, n).astype(np.uint32) if colours > 1 else None
    return _csr(n, rows), init


def make(spec: dict):
    """(off, idx, weight texts), init for a fixture entry's spec."""
    kind = spec["kind"]
    if kind == "known":
        return known(spec["name"])
    if kind == "lifted":
        return lifted(spec["seed"], spec["base_n"], spec["lift"], spec["pool_k"], spec["colours"])
    if kind == "random":
        return random_graph(spec["seed"], spec["n"], spec["max_deg"], spec["pool_k"], spec["colours"])
    raise KeyError(kind)


def specs():
    out = [{"kind": "known", "name": k} for k in KNOWN]
    for i in range(12):
        out.append({"kind": "lifted", "seed": 100 + i, "base_n": 6 + 3 * i, "lift": 2 + i % 7, "pool_k": 1 + i % 4,
                    "colours": 1 + i % 3})
    for i in range(8):
        out.append({"kind": "random", "seed": 200 + i, "n": 20 + 25 * i, "max_deg": 1 + i % 5, "pool_k": 1 + i % 3,
                    "colours": 1 + i % 2})
    # one larger case: 40,000 nodes
    out.append({"kind": "lifted", "seed": 300, "base_n": 400, "lift": 100, "pool_k": 3, "colours": 2})
    return out
