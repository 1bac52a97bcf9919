"""Generates tests/golden/law_cnr2000.json: the reference programs' results on
the reference's own LAW sample, cnr-2000 (webgraph-rs/data, BV-compressed;
325,557 nodes, 3,216,152 arcs), decoded by rbsc_b200's BV reader
(rbsc_bv_load) into oracle/_ref/cnr-2000.npz.

  * src/rsc/rsc.cpp            -> oracle/_ref/ref_rsc      (partition + rounds)
  * src/part_ref (Valmari)     -> oracle/_ref/ref_valmari  (exact partition)
  * src/rbsc/rbsc.cu           -> oracle/_ref/ref_rbsc     (`done`, `nodes`;
                                  --gpu, on a machine with a CUDA device)

Both CPU programs must agree (canonical partitions equal); the fixture keeps
checksums of the decoded CSR and of the canonical labels, the block count and
the round count (the GPU program's convention), and the programs' own
refinement times.  Uniform initial colours: the reference programs have none.

    python tests/golden/make_law_golden.py [--ref REFERENCE_CHECKOUT] [--gpu]
"""
from __future__ import annotations

import argparse
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

OUT = os.path.join(HERE, "law_cnr2000.json")


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: oracle.reference_tree())")
    ap.add_argument("--gpu", action="store_true", help="add the reference GPU program's output (needs a CUDA device)")
    args = ap.parse_args()
    args.ref = args.ref or oracle.reference_tree()
    if oracle.prepare_law(args.ref) is None:
        raise SystemExit("cnr-2000 not available (no reference tree, no decoded copy)")
    off, idx = oracle.load_law()
    fx = json.load(open(OUT)) if os.path.exists(OUT) else {}
    if not args.gpu:
        rs = oracle.run_ref_rsc(off, idx)
        vm = oracle.run_ref_valmari(off, idx)
        assert rs.blocks == vm.blocks and np.array_equal(rs.labels, vm.labels), "rsc and Valmari disagree"
        fx.update({"graph": "cnr-2000 (LAW, webgraph-rs/data of the reference)", "n": int(len(off) - 1),
                   "m": int(len(idx)), "csr_sha256": sha(off.astype(np.uint64), idx.astype(np.uint32)),
                   "blocks": int(rs.blocks), "rounds": int(rs.rounds), "rounds_cpu": int(rs.rounds_cpu),
                   "labels_sha256": sha(rs.labels.astype(np.uint32)),
                   "rsc_time_s": float(rs.time_s), "valmari_time_s": float(getattr(vm, "time_s", 0.0) or 0.0),
                   "sources": ["rsc", "valmari"]})
    else:
        # the reference GPU program at its bench's batch sizes (cuda, cuda_50, cuda_25)
        m = len(idx)
        runs = []
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "cnr.txt")
            oracle.write_arcs_file(path, off, idx)
            for exe, aggressive in ((oracle.REF_RBSC, False), (oracle.REF_RBSC + "_aggressive", True)):
                for b in (m, (m + 1) // 2, (m + 3) // 4):
                    if aggressive and b == m:
                        continue
                    with open(path, "rb") as f:
                        out = subprocess.run([exe, str(b), "1"], stdin=f, capture_output=True, timeout=900,
                                             check=True).stdout.decode()
                    lines = out.strip().splitlines()
                    runs.append({"batch": b, "aggressive": aggressive, "time_s": float(lines[0]), "done": int(lines[1]),
                                 "nodes": int(lines[2])})
        fx["ref_rbsc"] = {"runs": runs, "note": "the reference GPU programs (src/rbsc/rbsc.cu, rbsc_aggressive.cu, "
                                                "unmodified, sm_100a) run on a B200"}
    with open(OUT, "w") as f:
        json.dump(fx, f, indent=1)
    print(json.dumps(fx))


if __name__ == "__main__":
    main()
