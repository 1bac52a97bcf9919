"""The reference's own LAW sample, cnr-2000 (325,557 nodes, 3,216,152 arcs;
BV-compressed in the reference's webgraph-rs/data).

tests/golden/law_cnr2000.json (made by tests/golden/make_law_golden.py)
holds the reference programs' results on it: rsc and Valmari (partition,
blocks, rounds) and the reference GPU program's `done` / `nodes` at its
bench's batch sizes.  CPU: the BV reader against the format's own checks and
the fixture's checksum.  GPU: the CUDA path against the fixture (zero
tolerance), in one batch, in the reference's edge-batch mode, and streamed."""
import hashlib
import json
import os

import numpy as np
import pytest

import rbsc_b200 as R
from conftest import GOLDEN
from oracle import oracle

FX = json.load(open(os.path.join(GOLDEN, "law_cnr2000.json")))
_REF = oracle.reference_tree()
BV = os.path.join(_REF, "webgraph-rs", "data", "cnr-2000") if _REF else ""


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def law():
    g = oracle.load_law()
    if g is None:
        pytest.skip("decoded cnr-2000 not present (oracle/_ref/cnr-2000.npz is made by build() next to the reference)")
    off, idx = g
    assert _sha(off.astype(np.uint64), idx.astype(np.uint32)) == FX["csr_sha256"]
    return off, idx


@pytest.mark.skipif(not BV or not os.path.exists(BV + ".graph"),
                    reason="reference checkout not found ($RBSC_REFERENCE, else the location oracle/Makefile names)")
def test_bv_reader_on_the_reference_sample():
    off, idx, st = R.load_bvgraph(BV)
    assert len(off) - 1 == FX["n"] and len(idx) == FX["m"]
    assert _sha(off.astype(np.uint64), idx.astype(np.uint32)) == FX["csr_sha256"]
    # the compressor's own statistics (cnr-2000.properties) and list offsets
    props = dict(l.strip().split("=", 1) for l in open(BV + ".properties") if "=" in l and not l.startswith("#"))
    assert st["copied_arcs"] == int(props["copiedarcs"])
    assert st["interval_arcs"] == int(props["intervalisedarcs"])
    assert st["residual_arcs"] == int(props["residualarcs"])
    assert st["offsets_checked"] == 1
    # the transposed graph decodes to the transpose
    offt, idxt, _ = R.load_bvgraph(BV + "-t")
    n = len(off) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    order = np.lexsort((src, idx.astype(np.int64)))
    assert np.array_equal(idx.astype(np.int64)[order], np.repeat(np.arange(n), np.diff(offt.astype(np.int64))))
    assert np.array_equal(src[order], idxt.astype(np.int64))


def test_bv_reader_rejects_bad_input(tmp_path):
    base = str(tmp_path / "g")
    with open(base + ".properties", "w") as f:
        f.write("nodes=3\narcs=2\nwindowsize=7\nminintervallength=4\nzetak=3\ncompressionflags=OUTDEGREES_DELTA\n")
    open(base + ".graph", "wb").write(b"\x00")
    with pytest.raises(R.RbscError):
        R.load_bvgraph(base)
    with open(base + ".properties", "w") as f:
        f.write("nodes=3\narcs=2\nwindowsize=7\nminintervallength=4\nzetak=3\ncompressionflags=\n")
    open(base + ".graph", "wb").write(b"\xff")  # three empty lists: 0 arcs, not 2
    with pytest.raises(R.RbscError):
        R.load_bvgraph(base)


@pytest.mark.gpu
def test_gpu_partition_equals_the_reference_programs(law):
    off, idx = law
    with R.Context(0) as ctx:
        r = ctx.refine(off, idx)
        assert r.blocks == FX["blocks"] and r.rounds == FX["rounds"] and r.done == 1
        assert _sha(r.labels.astype(np.uint32)) == FX["labels_sha256"]
        g = ctx.upload(off, idx)
        for _ in range(2):
            r2 = g.refine()
            assert r2.blocks == FX["blocks"] and r2.rounds == FX["rounds"]
            assert _sha(r2.labels.astype(np.uint32)) == FX["labels_sha256"]
        g.free()


@pytest.mark.gpu
def test_gpu_edge_batches_equal_the_reference_gpu_program(law):
    off, idx = law
    with R.Context(0) as ctx:
        for run in FX["ref_rbsc"]["runs"]:
            r, info = ctx.refine_edge_batches(off, idx, edge_batch_size=run["batch"], aggressive=run["aggressive"],
                                              labels=False)
            assert (r.done, r.blocks) == (run["done"], run["nodes"]), run


@pytest.mark.gpu
def test_gpu_streamed_equals_the_reference_programs(law):
    off, idx = law
    with R.Context(0) as ctx:
        g = ctx.upload_streamed(off, idx, batch_arcs=len(idx) // 4 + 1)
        r = g.refine()
        g.free()
    assert r.blocks == FX["blocks"] and r.rounds == FX["rounds"]
    assert _sha(r.labels.astype(np.uint32)) == FX["labels_sha256"]


def _copy_bv(tmp_path, name, drop_offsets=False, drop_maxref=False, flip_at=None):
    import shutil
    dst = str(tmp_path / name)
    for ext in (".graph", ".properties", ".offsets"):
        if ext == ".offsets" and drop_offsets:
            continue
        shutil.copyfile(BV + ext, dst + ext)
    if drop_maxref:
        lines = [l for l in open(dst + ".properties") if not l.startswith("maxrefcount")]
        open(dst + ".properties", "w").write("".join(lines))
    if flip_at is not None:
        raw = bytearray(open(dst + ".graph", "rb").read())
        raw[int(len(raw) * flip_at)] ^= 0xff
        open(dst + ".graph", "wb").write(bytes(raw))
    return dst


@pytest.mark.skipif(not BV or not os.path.exists(BV + ".graph"),
                    reason="reference checkout not found ($RBSC_REFERENCE, else the location oracle/Makefile names)")
def test_bv_reader_paths_agree(tmp_path):
    """The threaded reader (offsets file and maxrefcount present: lists
    decoded by node ranges) and the one-pass reader (no offsets file, or no
    recorded maxrefcount) give the same CSR and statistics."""
    ref = R.load_bvgraph(BV)
    for kw in ({"drop_offsets": True}, {"drop_maxref": True}):
        off, idx, st = R.load_bvgraph(_copy_bv(tmp_path, "one_pass_" + "_".join(kw), **kw))
        assert np.array_equal(off, ref[0]) and np.array_equal(idx, ref[1])
        for k in ("copied_arcs", "interval_arcs", "residual_arcs", "bits"):
            assert st[k] == ref[2][k]
        assert st["offsets_checked"] == (0 if "drop_offsets" in kw else 1)


@pytest.mark.skipif(not BV or not os.path.exists(BV + ".graph"),
                    reason="reference checkout not found ($RBSC_REFERENCE, else the location oracle/Makefile names)")
@pytest.mark.parametrize("flip_at", [0.31, 0.77])
def test_bv_reader_rejects_a_corrupted_stream(tmp_path, flip_at):
    for kw in ({}, {"drop_maxref": True}):
        with pytest.raises(R.RbscError):
            R.load_bvgraph(_copy_bv(tmp_path, f"bad_{flip_at}_{len(kw)}", flip_at=flip_at, **kw))


@pytest.mark.skipif(not BV or not os.path.exists(BV + ".graph"),
                    reason="reference checkout not found ($RBSC_REFERENCE, else the location oracle/Makefile names)")
def test_cli_reads_bv_files(tmp_path):
    """`rbsc --bv BASENAME` loads the graph from the BV files instead of
    stdin (with --csr-cache the cache is written from them); without a GPU the
    command stops after loading, at the device."""
    import subprocess
    import torch
    cli = os.path.join(os.path.dirname(R.__file__), "rbsc")
    cache = str(tmp_path / "cnr.csr")
    r = subprocess.run([cli, "0", "1", "--bv", BV + ".graph", "--csr-cache", cache], capture_output=True, timeout=600)
    if torch.cuda.is_available():
        lines = r.stdout.decode().split()
        assert r.returncode == 0 and lines[1] == "1" and int(lines[2]) == FX["blocks"]
    else:
        assert r.returncode != 0 and b"CUDA setup failed" in r.stdout
    off, idx, wt = R.load_csr(cache)
    assert wt is None and _sha(off.astype(np.uint64), idx.astype(np.uint32)) == FX["csr_sha256"]
    r = subprocess.run([cli, "--bv", str(tmp_path / "missing")], capture_output=True, timeout=60)
    assert r.returncode != 0 and b"input error" in r.stdout
