"""Generates the golden fixtures of tests/golden/ by running the reference's own
programs, compiled unmodified from the reference tree by oracle/Makefile:

  * src/rsc/rsc.cpp            -> oracle/_ref/ref_rsc      (partition + rounds)
  * src/part_ref (Valmari)     -> oracle/_ref/ref_valmari  (exact partition)

For every case both reference programs must agree (canonical partitions equal,
same block count); the fixture then records the graph (or the generator call
that makes it, with a checksum), the canonical labels (or their checksum), the
block count and the round count reported by rsc (converted to the GPU
program's convention, rbsc.cu:339).

Run from the repository root (needs the reference tree: --ref, else $RBSC_REFERENCE, else the
location oracle/Makefile names):

    python tests/golden/make_golden.py [--ref REFERENCE_CHECKOUT]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from rbsc_b200 import graphs as G  # noqa: E402


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def weighted_case():
    """Nodes 0..7.  0 and 1 reach block {4,5} with total weight 3 (1+2 vs 3),
    2 reaches it with 2+2: lumpability sums weights per block."""
    s = [0, 0, 1, 2, 2, 3, 4, 5, 6]
    d = [4, 5, 4, 4, 5, 6, 7, 7, 7]
    w = [1, 2, 3, 2, 2, 1, 5, 5, 1]
    off, idx, wt = G.csr_from_arcs(8, s, d, w)
    return off, idx, wt


def cases():
    out = []
    out.append(("cycle7", *G.cycle(7), None, None))
    out.append(("path6", *G.path(6), None, None))
    out.append(("star9", *G.star_out(9), None, None))
    out.append(("bipartite3x4", *G.complete_bipartite(3, 4), None, None))
    out.append(("triangles_vs_hexagon", *G.two_triangles_and_hexagon(), None, None))
    u_off, u_idx, _ = G.disjoint_union([G.cycle(5), G.cycle(5), G.path(4), (np.zeros(4, np.uint64), np.zeros(0, np.uint32))])
    out.append(("union_cycles_path_isolated", u_off, u_idx, None, None))
    off, idx, wt = weighted_case()
    out.append(("weighted8", off, idx, wt, None))
    out.append(("lift64x8", *G.random_lift(64, 256, 8, seed=7), None, None))
    out.append(("er300", *G.er_directed(300, 1200, seed=11), None, None))
    out.append(("rmat10", *G.rmat(10, 8, seed=5), None, None))
    out.append(("regular3_40", *G.random_regular(40, 3, seed=3), None, None))
    off, idx = G.er_undirected(120, 4.0, seed=9)
    init = np.random.default_rng(9).integers(1, 9, size=120).astype(np.uint32)
    out.append(("er120_labels", off, idx, None, init))
    off, idx = G.rmat(9, 4, seed=2)
    init = np.asarray(np.diff(off.astype(np.int64)) > 2, dtype=np.uint32)
    out.append(("rmat9_degclass", off, idx, None, init))
    return out


# Larger cases are regenerated by the tests from their generator call; the
# fixture keeps checksums of the graph and of the expected labels.
GENERATED = [
    ("lift_4096x32", "random_lift", dict(base_n=4096, base_m=32768, lift=32, seed=1)),
    ("rmat14", "rmat", dict(scale=14, edge_factor=16, seed=1)),
]


def run_both(off, idx, wt, init):
    val = oracle.run_ref_valmari(off, idx, wt, init)
    rsc = None
    if init is None:
        rsc = oracle.run_ref_rsc(off, idx, wt)
        assert np.array_equal(rsc.labels, val.labels), "rsc and Valmari disagree"
        assert rsc.blocks == val.blocks
    return rsc, val


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: oracle.reference_tree())")
    args = ap.parse_args()
    args.ref = args.ref or oracle.reference_tree()
    oracle.build(ref=args.ref)
    index = {}
    for name, off, idx, wt, init in cases():
        rsc, val = run_both(off, idx, wt, init)
        arrays = dict(off=off.astype(np.uint64), idx=idx.astype(np.uint32), labels=val.labels.astype(np.uint32))
        if wt is not None:
            arrays["wt"] = wt.astype(np.uint64)
        if init is not None:
            arrays["init"] = init.astype(np.uint32)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        index[name] = dict(kind="arrays", n=len(off) - 1, m=int(off[-1]), blocks=val.blocks,
                           rounds=None if rsc is None else rsc.rounds, rounds_cpu=None if rsc is None else rsc.rounds_cpu,
                           sources=["valmari"] + ([] if rsc is None else ["rsc"]))
        print(name, index[name])
    for name, fn, kw in GENERATED:
        off, idx = getattr(G, fn)(**kw)
        rsc, val = run_both(off, idx, None, None)
        index[name] = dict(kind="generated", generator=fn, kwargs=kw, n=len(off) - 1, m=int(off[-1]),
                           graph_sha256=sha(off.astype(np.uint64), idx.astype(np.uint32)),
                           labels_sha256=sha(val.labels.astype(np.uint32)), blocks=val.blocks, rounds=rsc.rounds,
                           rounds_cpu=rsc.rounds_cpu, sources=["valmari", "rsc"])
        print(name, index[name])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
