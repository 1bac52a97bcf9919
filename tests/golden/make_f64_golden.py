"""Generates tests/golden/f64.json: the double-weight lumping fixtures.

Every case of f64_cases.specs() goes through Valmari's minimiser built with
double weights (src/part_ref/MDP_minimize.cc + MDP_read.cc, unmodified, with
MDP_weight_is_double: oracle/_ref/ref_valmari_f64, built by oracle/Makefile)
and through the oracle's restatement (oracle.c: orc_refine_f64, on the
doubles the minimiser's reader makes of the same decimal strings); the two
canonical partitions must be equal.  The fixture records, per case, the spec
that regenerates it, the checksum of the canonical labels, the block count and
the oracle's round count (passes until the count stopped changing).

Run from the repository root after `make -C oracle`:

    python tests/golden/make_f64_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import oracle  # noqa: E402
import f64_cases  # noqa: E402


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main():
    out = []
    for spec in f64_cases.specs():
        (off, idx, texts), init = f64_cases.make(spec)
        w = oracle.reader_decimals(texts)
        ref = oracle.run_ref_valmari_f64(off, idx, texts, init)
        orc = oracle.refine_f64(off, idx, w, init)
        if ref.blocks != orc.blocks or not np.array_equal(ref.labels, orc.labels):
            raise SystemExit(f"reference and oracle disagree on {spec}: {ref.blocks} vs {orc.blocks} blocks")
        entry = dict(spec)
        entry.update({"n": int(len(off) - 1), "m": int(off[-1]), "blocks": int(orc.blocks), "rounds": int(orc.rounds),
                      "labels_sha256": sha(orc.labels), "source": "ref_valmari_f64"})
        out.append(entry)
        print(entry["kind"], entry.get("name", entry.get("seed")), entry["n"], entry["m"], entry["blocks"], entry["rounds"])
    with open(os.path.join(HERE, "f64.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
