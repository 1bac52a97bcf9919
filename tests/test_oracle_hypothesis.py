"""Property-based cross-check of the oracle on tiny random graphs (hypothesis
draws the graphs): the exact refinement, the rsc restatement (serial and on
threads) and, where built, the unmodified Valmari program give the same
partition, and the exact partition is stable and refines the initial
colours."""
import os

import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings, strategies as st

from oracle import oracle
from rbsc_b200 import graphs as G


@st.composite
def graphs(draw):
    n = draw(st.integers(1, 24))
    m = draw(st.integers(0, 60))
    src = np.array(draw(st.lists(st.integers(0, n - 1), min_size=m, max_size=m)), dtype=np.int64)
    dst = np.array(draw(st.lists(st.integers(0, n - 1), min_size=m, max_size=m)), dtype=np.int64)
    weighted = draw(st.booleans())
    wt = np.array(draw(st.lists(st.integers(1, 4), min_size=m, max_size=m)), dtype=np.uint64) if weighted else None
    colours = draw(st.integers(1, 3))
    init = np.array(draw(st.lists(st.integers(0, colours - 1), min_size=n, max_size=n)), dtype=np.uint32)
    off, idx, w = G.csr_from_arcs(n, src, dst, wt)
    return off, idx, w, init


def _stable(off, idx, wt, init, labels):
    """Every block is uniform in the initial colour, and its members have the
    same weight sum into every block."""
    n = len(off) - 1
    for u in range(n):
        for v in range(n):
            if labels[u] != labels[v]:
                continue
            if init[u] != init[v]:
                return False
            su, sv = {}, {}
            for s, x in ((su, u), (sv, v)):
                for k in range(int(off[x]), int(off[x + 1])):
                    b = int(labels[idx[k]])
                    s[b] = s.get(b, 0) + (int(wt[k]) if wt is not None else 1)
            if su != sv:
                return False
    return True


@settings(max_examples=200, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(graphs())
def test_oracles_agree_on_tiny_graphs(g):
    off, idx, wt, init = g
    ex = oracle.refine_exact(off, idx, wt, init)
    rs = oracle.refine_rsc(off, idx, wt, init)
    mt = oracle.refine_rsc(off, idx, wt, init, threads=3)
    assert np.array_equal(ex.labels, rs.labels) and ex.blocks == rs.blocks and ex.rounds == rs.rounds
    assert np.array_equal(rs.labels, mt.labels) and rs.rounds_cpu == mt.rounds_cpu
    assert _stable(off, idx, wt, init, ex.labels)
    if os.path.exists(oracle.REF_VALMARI):
        val = oracle.run_ref_valmari(off, idx, wt, init)
        assert np.array_equal(ex.labels, val.labels) and ex.blocks == val.blocks
