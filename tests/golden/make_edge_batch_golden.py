"""Generates tests/golden/edge_batches.json by running the reference's own GPU
program in its edge-batch mode: src/rbsc/rbsc.cu and src/rbsc/rbsc_aggressive.cu
compiled unmodified by oracle/Makefile into oracle/_ref/ref_rbsc and
oracle/_ref/ref_rbsc_aggressive.

For every (graph, edge_batch_size) case the fixture records the two values
the reference prints besides its time: `done` and `nodes` (rbsc.cu:493-494),
for the plain and the aggressive program.  The graphs are regenerated by the
tests from the generator calls recorded here (rbsc_b200.graphs, seeded numpy),
with a checksum of the arcs.

Needs a CUDA device (the reference program runs on it).  Run from the
repository root:

    python tests/golden/make_edge_batch_golden.py
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from rbsc_b200 import graphs as G  # noqa: E402

REF_RBSC = os.path.join(ROOT, "oracle", "_ref", "ref_rbsc")
REF_RBSC_AGGR = os.path.join(ROOT, "oracle", "_ref", "ref_rbsc_aggressive")

# (name, generator in rbsc_b200.graphs, kwargs)
GRAPHS = [
    ("cycle7", "cycle", dict(n=7)),
    ("path6", "path", dict(n=6)),
    ("star9", "star_out", dict(n=9)),
    ("lift64x8", "random_lift", dict(base_n=64, base_m=256, lift=8, seed=7)),
    ("lift128x4", "random_lift", dict(base_n=128, base_m=640, lift=4, seed=3)),
    ("er300", "er_directed", dict(n=300, m=1200, seed=11)),
    ("er2000", "er_directed", dict(n=2000, m=6000, seed=5)),
    ("rmat10", "rmat", dict(scale=10, edge_factor=8, seed=5)),
    ("rmat12", "rmat", dict(scale=12, edge_factor=4, seed=2)),
    ("regular3_40", "random_regular", dict(n=40, d=3, seed=3)),
    ("rmat14", "rmat", dict(scale=14, edge_factor=16, seed=1)),
]

# batch sizes as fractions of M (the reference's cuda_50 / cuda_25 columns and
# smaller), plus a fixed small size on the small graphs
FRACTIONS = [1.0, 0.5, 0.25, 0.1]
FIXED = [100]


def graph(gen: str, kw: dict):
    return getattr(G, gen)(**kw)


def sha(off, idx) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(idx, dtype=np.uint32).tobytes())
    return h.hexdigest()


def run_ref(exe: str, path: str, batch: int):
    """(done, nodes) printed by the reference, or None if it did not finish
    within 120 s (such cases are left out of the fixture)."""
    with open(path, "rb") as f:
        try:
            out = subprocess.run([exe, str(batch), "1"], stdin=f, capture_output=True, timeout=120,
                                 check=True).stdout.decode()
        except subprocess.TimeoutExpired:
            return None
    lines = out.strip().splitlines()
    return int(lines[1]), int(lines[2])


def main():
    for exe in (REF_RBSC, REF_RBSC_AGGR):
        if not os.path.exists(exe):
            raise SystemExit(f"{exe} not built (make -C oracle with the reference tree present)")
    cases = []
    with tempfile.TemporaryDirectory() as d, cf.ThreadPoolExecutor(8) as pool:
        jobs = []
        for name, gen, kw in GRAPHS:
            off, idx = graph(gen, kw)
            m = len(idx)
            path = os.path.join(d, f"{name}.txt")
            oracle.write_arcs_file(path, off, idx)
            sizes = sorted({max(1, int(round(f * m))) for f in FRACTIONS} | {b for b in FIXED if b < m <= 2000})
            for b in sizes:
                case = dict(graph=name, generator=gen, kwargs=kw, n=len(off) - 1, m=m, sha256=sha(off, idx), batch=b)
                jobs.append((case, pool.submit(run_ref, REF_RBSC, path, b), pool.submit(run_ref, REF_RBSC_AGGR, path, b)))
        for case, plain, aggr in jobs:
            if plain.result() is None or aggr.result() is None:
                print("timed out:", case["graph"], case["batch"], flush=True)
                continue
            case["done"], case["nodes"] = plain.result()
            case["done_aggressive"], case["nodes_aggressive"] = aggr.result()
            cases.append(case)
            print(case["graph"], case["m"], case["batch"], case["done"], case["nodes"], case["done_aggressive"],
                  case["nodes_aggressive"], flush=True)
    with open(os.path.join(HERE, "edge_batches.json"), "w") as f:
        json.dump({"source": "oracle/_ref/ref_rbsc and ref_rbsc_aggressive (src/rbsc/rbsc.cu, rbsc_aggressive.cu "
                             "compiled unmodified), run on a B200", "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
