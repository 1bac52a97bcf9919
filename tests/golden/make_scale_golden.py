"""Generates tests/golden/scale.json: oracle results at the benchmark
configurations' own sizes, for the GPU tests in tests/test_scale_parity.py.

  rmat24_ef16   the plain-refinement-at-scale workload: R-MAT scale 24, edge
                factor 16, (a, b, c) = (0.57, 0.19, 0.19), seed 1, duplicates and
                self-loops removed, initial colours floor(log2(out_degree+1)).
                Three oracles must agree on the partition:
                  * Valmari's exact minimiser (src/part_ref, unmodified) with the
                    initial colours as MDP <blocks> (MDP_read.cc:140-150);
                  * the reference rsc (src/rsc/rsc.cpp, unmodified), which fixes
                    uniform initial colours (rsc.cpp:118-121): the degree
                    classes are implied by the graph's structure after one round,
                    so its final partition is the same;
                  * the restatement of rsc's loop with the initial colours
                    (oracle.c: orc_refine_rsc_mt), which gives the round count
                    in the GPU program's convention (rbsc.cu:339).
  wl_batch_100k the small-graph batch: 100,000 graphs, n ~ U[10, 500], half
                Erdos-Renyi (mean degree 4), half random 3-regular, labels
                U{1..8}, seed 1, side by side.  Oracles: Valmari with the labels
                as <blocks>, and orc_refine_rsc_mt (round count).  rsc cannot take
                initial colours, and the labels are not implied by structure.
  rmat28_ef32   (--only rmat28; needs a GPU and about 80 GB of host memory)
                the out-of-HBM workload: R-MAT scale 28, edge factor 32, seed 1,
                generated on the device into page-locked host memory by the
                product's generator; degree-bucket initial colours.  Neither
                reference program takes it (rsc's total weight limit 2^32-1,
                rsc.cpp:17-23; Valmari's 32-bit counts), so the oracle is
                orc_refine_rsc_mt with 64-bit counters, run on the host cores.

Each entry records the input's checksum (so a test knows it regenerated the
same input), the sha256 of the canonical labels (uint32, smallest node id of
each block), the block count and the round count.

Run from the repository root, with the reference programs built
(RBSC_REFERENCE=<reference checkout> python -c "import __graft_entry__ as g; g.build()"):

    python tests/golden/make_scale_golden.py [--only rmat24|batch|rmat28]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

OUT = os.path.join(HERE, "scale.json")


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        step = 1 << 28
        flat = a.reshape(-1).view(np.uint8)
        for i in range(0, flat.size, step):
            h.update(flat[i: i + step])
    return h.hexdigest()


def degree_colours(off) -> np.ndarray:
    """floor(log2(out_degree + 1)) as uint32 (bit length of out_degree + 1, less one)."""
    x = np.diff(np.asarray(off, dtype=np.int64)) + 1
    out = np.zeros(x.shape, dtype=np.uint32)
    for sh in (32, 16, 8, 4, 2, 1):
        big = x >= (1 << sh)
        out[big] += sh
        x = np.where(big, x >> sh, x)
    return out


def parse_labels(txt: str) -> np.ndarray:
    i = txt.index("labels")
    line = txt[i + 6: txt.index("\n", i)]
    return np.array(line.split(), dtype=np.uint64)


def canon(labels_u64) -> np.ndarray:
    _, inv = np.unique(labels_u64, return_inverse=True)
    return oracle.canonicalize(inv.astype(np.uint32))[0]


def run_rsc(off, idx, d):
    path = os.path.join(d, "arcs.txt")
    oracle.write_arcs_file(path, off, idx)
    t0 = time.time()
    with open(path, "rb") as f:
        txt = subprocess.run([oracle.REF_RSC], stdin=f, capture_output=True, check=True).stdout.decode()
    os.unlink(path)
    lines = txt.split("\n")
    rounds_cpu = int(next(ln for ln in lines if ln.startswith("rounds ")).split()[1])
    lab = canon(parse_labels(txt))
    print(f"  rsc: {time.time() - t0:.1f} s, refinement {float(lines[0]):.2f} s, blocks {lines[2]}, rounds {rounds_cpu}",
          flush=True)
    return lab, int(lines[2]), rounds_cpu


def run_valmari(off, idx, init, d):
    path = os.path.join(d, "mdp.txt")
    oracle.write_mdp_file(path, off, idx, init=init)
    t0 = time.time()
    with open(path, "rb") as f:
        txt = subprocess.run([oracle.REF_VALMARI], stdin=f, capture_output=True, check=True).stdout.decode()
    os.unlink(path)
    lines = txt.split("\n")
    lab = canon(parse_labels(txt))
    blocks = int(np.unique(lab).size)
    print(f"  valmari: {time.time() - t0:.1f} s, blocks {blocks} ({lines[:3]})", flush=True)
    return lab, blocks


def run_mt(off, idx, init, threads):
    t0 = time.time()
    r = oracle.refine_rsc(off, idx, init=init, threads=threads)
    assert r.status == 0, r.status
    print(f"  rsc restatement ({threads} threads): {time.time() - t0:.1f} s, blocks {r.blocks}, "
          f"rounds {r.rounds} (cpu convention {r.rounds_cpu})", flush=True)
    return r


def case_rmat24(threads, scale=24):
    print(f"rmat{scale}_ef16", flush=True)
    off, idx = oracle.gen_rmat(scale, 16, seed=1, threads=threads)
    init = degree_colours(off)
    with tempfile.TemporaryDirectory() as d:
        lab_v, blocks_v = run_valmari(off, idx, init, d)
        lab_r, blocks_r, rounds_cpu = run_rsc(off, idx, d)
    mt = run_mt(off, idx, init, threads)
    assert np.array_equal(lab_v, lab_r) and blocks_v == blocks_r, "rsc and Valmari disagree"
    assert np.array_equal(lab_v, mt.labels) and blocks_v == mt.blocks, "restatement and Valmari disagree"
    return dict(kind="rmat", scale=scale, edge_factor=16, seed=1, initial_colours="floor(log2(out_degree+1))",
                n=len(off) - 1, m=int(off[-1]), graph_sha256=sha(off.astype(np.uint64), idx.astype(np.uint32)),
                labels_sha256=sha(lab_v.astype(np.uint32)), blocks=blocks_v, rounds=mt.rounds,
                rounds_cpu_uniform_start=rounds_cpu, sources=["valmari", "rsc", "rsc_restatement"])


def case_batch(threads, graphs=100000):
    print(f"wl_batch_{graphs}", flush=True)
    import rbsc_b200 as R  # the batch generator (input only; the oracles check the result)
    off, idx, gn, lab = R.gen_wl_batch(graphs, 10, 500, 8, seed=1)
    with tempfile.TemporaryDirectory() as d:
        lab_v, blocks_v = run_valmari(off, idx, lab, d)
    mt = run_mt(off, idx, lab, threads)
    assert np.array_equal(lab_v, mt.labels) and blocks_v == mt.blocks, "restatement and Valmari disagree"
    # per-graph block counts: distinct union labels inside each graph's node range
    G = len(gn) - 1
    gid = np.repeat(np.arange(G, dtype=np.int64), np.diff(gn.astype(np.int64)))
    pairs = np.unique(gid * (1 << 32) + lab_v.astype(np.int64))
    per_graph = np.bincount((pairs >> 32).astype(np.int64), minlength=G).astype(np.uint32)
    return dict(kind="wl_batch", graphs=graphs, nmin=10, nmax=500, num_labels=8, seed=1,
                n=len(off) - 1, m=int(off[-1]),
                graph_sha256=sha(off.astype(np.uint64), idx.astype(np.uint32), gn.astype(np.uint64),
                                 lab.astype(np.uint32)),
                labels_sha256=sha(lab_v.astype(np.uint32)), blocks=blocks_v, rounds=mt.rounds,
                per_graph_blocks_sha256=sha(per_graph), sources=["valmari", "rsc_restatement"])


def case_rmat28(threads):
    print("rmat28_ef32", flush=True)
    import rbsc_b200 as R  # the device generator writes the arcs into page-locked host memory
    t0 = time.time()
    with R.Context(0) as ctx:
        pg = ctx.gen_rmat_pinned(28, 32, seed=1)
        off, idx = pg.off, pg.idx
        print(f"  generated {len(idx)} arcs in {time.time() - t0:.1f} s", flush=True)
        init = degree_colours(off)
        mt = run_mt(off, idx, init, threads)
        entry = dict(kind="rmat_pinned", scale=28, edge_factor=32, seed=1,
                     initial_colours="floor(log2(out_degree+1))", n=len(off) - 1, m=int(len(idx)),
                     offsets_sha256=sha(np.asarray(off, dtype=np.uint64)),
                     labels_sha256=sha(mt.labels.astype(np.uint32)), blocks=mt.blocks, rounds=mt.rounds,
                     sources=["rsc_restatement"])
        pg.free()
    return entry


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["rmat24", "batch", "rmat28"], action="append")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    which = args.only or ["rmat24", "batch"]
    index = json.load(open(OUT)) if os.path.exists(OUT) else {}
    fns = {"rmat24": ("rmat24_ef16", case_rmat24), "batch": ("wl_batch_100k", case_batch),
           "rmat28": ("rmat28_ef32", case_rmat28)}
    for w in which:
        name, fn = fns[w]
        t0 = time.time()
        index[name] = fn(args.threads)
        index[name]["generated_in_s"] = round(time.time() - t0, 1)
        print(name, index[name], flush=True)
        with open(OUT, "w") as f:
            json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
