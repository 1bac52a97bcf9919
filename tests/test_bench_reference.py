"""The bench's reference arm (`bench.py --impl reference`): the unmodified
reference rsc program timed on the host cores, printed as one JSON line with
the same metric, unit and config as the GPU arm.  Runs on the CPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference program was not built here
        return
    assert d["metric"].startswith("edge-rounds/s") and d["unit"] == "edge-rounds/s"
    assert d["value"] > 0 and d["steps"] == 1 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "rmat24_ef16"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_cpu_baseline_has_the_reference_and_an_all_cores_port():
    """The GPU arm's cpu_baseline leg, run here on the CPU: the reference
    program on one core, and the oracle's threaded rsc restatement on every
    core over the same sample with the same rounds and blocks."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.cpu_baseline_reference()
    assert c["value"] > 0 and c["unit"] == "edge-rounds/s" and c["cores"] == 1
    p = c["port_all_cores"]
    assert "unavailable" not in p, p
    assert p["kind"] == "port" and p["cores"] == (os.cpu_count() or 1) and p["value"] > 0
    if c["kind"] == "reference":
        assert p["rounds"] == c["runs"][0]["rounds"] and p["blocks"] == c["runs"][0]["blocks"]
