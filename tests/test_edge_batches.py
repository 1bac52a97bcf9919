"""The reference's edge-batch (quotient) mode, rbsc.cu:292-487 and the stop
test of rbsc_aggressive.cu:487.

tests/golden/edge_batches.json holds what the reference's own GPU programs
print (`done`, `nodes`) for seeded graphs and batch sizes (made by
tests/golden/make_edge_batch_golden.py).  CPU: the oracle's restatement
(oracle.c: orc_refine_edge_batches) reproduces every case.  GPU: the CUDA
path (rbsc_refine_edge_batches) gives the same counts and the oracle's exact
final partition.  Integer work: no tolerance."""
import json
import os

import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import graphs as G
from conftest import GOLDEN
from oracle import oracle

with open(os.path.join(GOLDEN, "edge_batches.json")) as f:
    CASES = json.load(f)["cases"]

_graphs = {}


def _graph(c):
    key = c["graph"]
    if key not in _graphs:
        _graphs[key] = getattr(G, c["generator"])(**c["kwargs"])
    return _graphs[key]


def _ids(c):
    return f"{c['graph']}-b{c['batch']}"


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_oracle_matches_reference(case):
    off, idx = _graph(case)
    assert len(off) - 1 == case["n"] and len(idx) == case["m"]
    r = oracle.refine_edge_batches(off, idx, batch=case["batch"])
    assert (r.done, r.blocks) == (case["done"], case["nodes"])
    ra = oracle.refine_edge_batches(off, idx, batch=case["batch"], aggressive=True)
    assert (ra.done, ra.blocks) == (case["done_aggressive"], case["nodes_aggressive"])


def test_oracle_one_batch_is_the_exact_partition():
    off, idx = G.rmat(10, 8, seed=5)
    r = oracle.refine_edge_batches(off, idx, batch=len(idx))
    ex = oracle.refine_exact(off, idx)
    assert r.done == 1 and r.iterations == 1 and r.blocks == ex.blocks
    assert np.array_equal(r.labels, ex.labels)


def test_oracle_batches_refine_the_coarsest_partition():
    """A batched result is finer than or equal to the coarsest partition."""
    off, idx = G.random_lift(64, 256, 8, seed=7)
    ex = oracle.refine_exact(off, idx)
    for b in (100, 500, 1000):
        r = oracle.refine_edge_batches(off, idx, batch=b)
        # every block of r lies inside one block of ex
        pairs = set(zip(r.labels.tolist(), ex.labels.tolist()))
        assert len(pairs) == len(set(r.labels.tolist()))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_gpu_matches_reference(case):
    off, idx = _graph(case)
    with R.Context(0) as ctx:
        r, info = ctx.refine_edge_batches(off, idx, edge_batch_size=case["batch"])
        ra, _ = ctx.refine_edge_batches(off, idx, edge_batch_size=case["batch"], aggressive=True)
    assert (r.done, r.blocks) == (case["done"], case["nodes"])
    assert (ra.done, ra.blocks) == (case["done_aggressive"], case["nodes_aggressive"])
    ex = oracle.refine_edge_batches(off, idx, batch=case["batch"])
    assert np.array_equal(r.labels, ex.labels)
    assert info["iterations"] == ex.iterations


@pytest.mark.gpu
def test_gpu_weighted_and_edge_cases():
    rng = np.random.default_rng(4)
    off, idx = G.er_directed(400, 2400, seed=8)
    wt = rng.integers(1, 4, size=len(idx)).astype(np.uint64)
    with R.Context(0) as ctx:
        for b in (len(idx), 600, 97):
            r, _ = ctx.refine_edge_batches(off, idx, wt, edge_batch_size=b)
            ex = oracle.refine_edge_batches(off, idx, wt, batch=b)
            assert (r.done, r.blocks) == (ex.done, ex.blocks) and np.array_equal(r.labels, ex.labels)
        # no arc at all: no batch, as the reference prints (nodes 0, done 0)
        r, _ = ctx.refine_edge_batches(np.zeros(6, np.uint64), np.zeros(0, np.uint32), edge_batch_size=4)
        assert (r.done, r.blocks) == (0, 0) and np.all(r.labels == 0)
        # a row longer than the batch: batch 0 is skipped, its node stays alone
        off, idx = G.star_out(40)
        r, _ = ctx.refine_edge_batches(off, idx, edge_batch_size=8)
        ex = oracle.refine_edge_batches(off, idx, batch=8)
        assert (r.done, r.blocks) == (ex.done, ex.blocks) and np.array_equal(r.labels, ex.labels)


@pytest.mark.gpu
def test_cli_edge_batch_size_matches_reference():
    """The `rbsc` command prints the reference's `done` / `nodes` for a batch size."""
    import subprocess
    from rbsc_b200._lib import CLI_PATH
    case = next(c for c in CASES if c["graph"] == "rmat12" and c["done"] == 0)
    off, idx = _graph(case)
    txt = oracle.arcs_cuda_text(off, idx)
    out = subprocess.run([CLI_PATH, str(case["batch"]), "1"], input=txt, capture_output=True, check=True).stdout.decode()
    lines = out.strip().splitlines()
    assert (int(lines[1]), int(lines[2])) == (case["done"], case["nodes"])
    out = subprocess.run([CLI_PATH, str(case["batch"]), "1", "--aggressive"], input=txt, capture_output=True,
                         check=True).stdout.decode()
    lines = out.strip().splitlines()
    assert (int(lines[1]), int(lines[2])) == (case["done_aggressive"], case["nodes_aggressive"])
