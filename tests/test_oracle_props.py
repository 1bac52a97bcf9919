"""Oracle self-consistency on random small graphs: the exact restatement, the
rsc restatement and (when built) the reference programs agree."""
import os

import numpy as np
import pytest

from oracle import oracle
from rbsc_b200 import graphs as G


def _graphs():
    yield "er", *G.er_directed(200, 600, seed=1)
    yield "lift", *G.random_lift(32, 96, 6, seed=2)
    yield "rmat", *G.rmat(8, 6, seed=3)
    yield "reg", *G.random_regular(30, 3, seed=4)
    yield "isolated", np.zeros(11, dtype=np.uint64), np.zeros(0, dtype=np.uint32)


@pytest.mark.parametrize("case", list(_graphs()), ids=lambda c: c[0])
def test_exact_equals_rsc_restatement(case):
    _, off, idx = case
    a = oracle.refine_exact(off, idx)
    b = oracle.refine_rsc(off, idx)
    assert np.array_equal(a.labels, b.labels)
    assert a.blocks == b.blocks and a.rounds == b.rounds


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_initial_colours_refine(seed):
    off, idx = G.er_undirected(80, 3.0, seed=seed)
    init = np.random.default_rng(seed).integers(0, 4, size=80).astype(np.uint32)
    a = oracle.refine_exact(off, idx, init=init)
    b = oracle.refine_rsc(off, idx, init=init)
    assert np.array_equal(a.labels, b.labels)
    # the result refines the initial colouring
    for blk in np.unique(a.labels):
        assert np.unique(init[a.labels == blk]).size == 1


def test_round_blocks_monotone():
    off, idx = G.rmat(9, 8, seed=5)
    r = oracle.refine_exact(off, idx)
    rb = r.round_blocks
    assert rb[0] == 1 and all(x <= y for x, y in zip(rb, rb[1:]))
    assert rb[-1] == rb[-2] == r.blocks


@pytest.mark.skipif(not os.path.exists(oracle.REF_VALMARI), reason="reference binaries not built")
def test_valmari_with_initial_blocks():
    off, idx = G.er_undirected(60, 3.0, seed=7)
    init = np.random.default_rng(7).integers(0, 3, size=60).astype(np.uint32)
    a = oracle.refine_exact(off, idx, init=init)
    v = oracle.run_ref_valmari(off, idx, init=init)
    assert np.array_equal(a.labels, v.labels)


def test_empty_graph():
    r = oracle.refine_exact(np.zeros(1, dtype=np.uint64), np.zeros(0, dtype=np.uint32))
    assert r.blocks == 0 and r.rounds == 0


def _mt_cases():
    import rbsc_b200 as R
    yield "er", *G.er_directed(300, 1200, seed=11), None, None
    off, idx = G.rmat(13, 8, seed=12)
    yield "rmat13_degree_colours", off, idx, None, R.degree_bucket_colors(off)
    off, idx = G.random_lift(64, 256, 8, seed=13)
    yield "lift_weighted", off, idx, np.random.default_rng(13).integers(1, 5, len(idx)).astype(np.uint64), None
    off, idx = G.er_undirected(500, 3.0, seed=14)
    yield "labels", off, idx, None, np.random.default_rng(14).integers(0, 6, 500).astype(np.uint32)
    yield "isolated", np.zeros(11, dtype=np.uint64), np.zeros(0, dtype=np.uint32), None, None
    yield "empty", np.zeros(1, dtype=np.uint64), np.zeros(0, dtype=np.uint32), None, None


@pytest.mark.parametrize("threads", [1, 3, 8])
@pytest.mark.parametrize("case", list(_mt_cases()), ids=lambda c: c[0])
def test_multithreaded_rsc_restatement_is_the_same(case, threads):
    """orc_refine_rsc_mt (for graphs of billions of arcs) gives the serial
    restatement's labels, blocks, rounds in both conventions and status."""
    _, off, idx, wt, init = case
    a = oracle.refine_rsc(off, idx, wt, init)
    b = oracle.refine_rsc(off, idx, wt, init, threads=threads)
    assert np.array_equal(a.labels, b.labels)
    assert (a.blocks, a.rounds, a.rounds_cpu, a.status) == (b.blocks, b.rounds, b.rounds_cpu, b.status)


@pytest.mark.parametrize("max_rounds", [0, 1, 2])
def test_multithreaded_rsc_restatement_stopped_early(max_rounds):
    off, idx = G.rmat(10, 8, seed=15)
    a = oracle.refine_rsc(off, idx, max_rounds=max_rounds)
    b = oracle.refine_rsc(off, idx, max_rounds=max_rounds, threads=4)
    assert np.array_equal(a.labels, b.labels) and a.blocks == b.blocks and a.status == b.status == -1
