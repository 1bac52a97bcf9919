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
