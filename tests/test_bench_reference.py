"""The bench's reference arm (`bench.py --impl reference`): the unmodified
reference rsc program timed on the host cores on the workload's own graph,
printed as one JSON line with the same metric, unit and config as the GPU arm,
without loading anything of the product.  Runs on the CPU, at a small scale."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_ARM = r"""
import sys
sys.argv = ["bench.py", "--impl", "reference", "--scale", "15", "--steps", "3", "--warmup", "1"]
sys.path.insert(0, ".")
import bench
rc = bench.main()
loaded = [m for m in sys.modules if m == "rbsc_b200" or m.startswith("rbsc_b200.")]
maps = open("/proc/self/maps").read()
print("PRODUCT_MODULES", loaded, "librbsc" in maps)
sys.exit(rc)
"""


def test_reference_arm_prints_one_contract_line_without_the_product():
    r = subprocess.run([sys.executable, "-c", _ARM], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert "PRODUCT_MODULES [] False" in r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference program was not built here
        return
    assert d["metric"].startswith("edge-rounds/s") and d["unit"] == "edge-rounds/s"
    assert d["value"] > 0 and d["steps"] == 3 and d["warmup"] == 1 and d["higher_is_better"] is True
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle
    off, idx = oracle.gen_rmat(15, 16, seed=1)
    # the same config object as the GPU arm prints for this graph
    assert d["config"] == json.loads(json.dumps(bench.config(len(off) - 1, len(idx), 15, 16)))
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the reference's block count is the exact one
    assert d["blocks"] == oracle.refine_exact(off, idx).blocks


def test_ref_rsc_round_samples_one_parse_several_runs():
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle
    if not os.path.exists(oracle.REF_RSC):
        return
    off, idx = oracle.gen_rmat(12, 8, seed=4)
    r = bench.ref_rsc_round_samples(off, idx, 7)
    assert len(r["round_s"]) >= 7 and all(t > 0 for t in r["round_s"])
    rounds = {x["rounds"] for x in r["runs"]}
    blocks = {x["blocks"] for x in r["runs"]}
    assert len(rounds) == 1 and len(blocks) == 1       # every forked run is the same refinement
    assert len(r["round_s"]) == len(r["runs"]) * (rounds.pop() - 1)
    assert blocks.pop() == oracle.refine_exact(off, idx).blocks


def test_cpu_baseline_has_the_reference_and_an_all_cores_port():
    """The GPU arm's cpu_baseline leg, run here on the CPU: the reference
    program on one core, and the oracle's threaded rsc restatement on every
    core over the same graph with the same rounds and blocks."""
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle
    off, idx = oracle.gen_rmat(14, 16, seed=1)
    c = bench.cpu_baseline_reference(off, idx, samples=2)
    assert c["value"] > 0 and c["unit"] == "edge-rounds/s"
    p = c["port_all_cores"]
    assert "unavailable" not in p, p
    assert p["kind"] == "port" and p["cores"] == (os.cpu_count() or 1) and p["value"] > 0
    if c["kind"] == "reference":
        assert c["cores"] == 1 and len(c["round_s"]) == 2
        assert p["rounds"] == c["rsc_own_timer"]["rounds"] and p["blocks"] == c["rsc_own_timer"]["blocks"]


def test_roofline_traffic_is_committed_for_every_first_pass_kernel():
    """The bench's roofline `traffic` comes from the committed R-MAT-24 ncu
    summary of the first pass's kernel (profiles/<kernel>_rmat24.md, line
    'traffic_bytes_per_arc: X'): each kernel the bench can name has one, with
    a per-arc figure in the range a gather of 1-byte ranks over 4-byte heads
    gives (below the 8 algorithmic bytes per arc)."""
    sys.path.insert(0, ROOT)
    import bench
    for kernel in ("k_signature", "k_signature_hot", "k_signature_hot_tma"):
        tpa = bench.signature_traffic_per_arc(kernel)
        assert tpa is not None, kernel
        assert 4.0 < tpa < 8.0, (kernel, tpa)
