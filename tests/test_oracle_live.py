"""The oracle against the unmodified reference programs, run live here (they
are built from the reference sources by oracle/Makefile): random graphs with
multi-arcs, self-loops, nodes without arcs, integer weights and initial
blocks.  Partitions (canonical labels) must be identical; rsc's round count,
converted to the GPU program's convention, must equal the oracle's."""
import os

import numpy as np
import pytest

from oracle import oracle
from rbsc_b200 import graphs as G

pytestmark = pytest.mark.skipif(not (os.path.exists(oracle.REF_RSC) and os.path.exists(oracle.REF_VALMARI)),
                                reason="reference programs not built")


def _messy(seed: int):
    """n nodes, arcs drawn with repetition (multi-arcs) from a skewed head
    distribution, some self-loops, a tail of nodes without arcs."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(30, 600))
    m = int(rng.integers(n, 6 * n))
    active = max(2, int(n * rng.uniform(0.5, 0.95)))  # nodes >= active have no arcs
    src = rng.integers(0, active, size=m)
    dst = np.minimum((rng.pareto(1.2, size=m) * 5).astype(np.int64), n - 1)
    loops = rng.random(m) < 0.05
    dst[loops] = src[loops]
    off, idx, _ = G.csr_from_arcs(n, src, dst)
    return off, idx


@pytest.mark.parametrize("seed", range(8))
def test_oracle_equals_rsc_and_valmari_unweighted(seed):
    off, idx = _messy(seed)
    ex = oracle.refine_exact(off, idx)
    rsc = oracle.run_ref_rsc(off, idx)
    val = oracle.run_ref_valmari(off, idx)
    assert np.array_equal(ex.labels, rsc.labels) and ex.blocks == rsc.blocks
    assert ex.rounds == rsc.rounds
    assert np.array_equal(ex.labels, val.labels) and ex.blocks == val.blocks


@pytest.mark.parametrize("seed", range(8, 14))
def test_oracle_equals_rsc_and_valmari_weighted(seed):
    off, idx = _messy(seed)
    wt = np.random.default_rng(seed).integers(1, 6, size=len(idx)).astype(np.uint64)
    ex = oracle.refine_exact(off, idx, wt)
    rsc = oracle.run_ref_rsc(off, idx, wt)
    val = oracle.run_ref_valmari(off, idx, wt)
    assert np.array_equal(ex.labels, rsc.labels) and ex.blocks == rsc.blocks
    assert np.array_equal(ex.labels, val.labels) and ex.blocks == val.blocks


@pytest.mark.parametrize("seed", range(14, 20))
def test_oracle_equals_valmari_with_initial_blocks(seed):
    off, idx = _messy(seed)
    n = len(off) - 1
    init = np.random.default_rng(seed).integers(0, 5, size=n).astype(np.uint32)
    ex = oracle.refine_exact(off, idx, init=init)
    val = oracle.run_ref_valmari(off, idx, init=init)
    assert np.array_equal(ex.labels, val.labels) and ex.blocks == val.blocks


@pytest.mark.parametrize("seed", range(20, 24))
def test_valmari_input_with_parallel_arcs_merged_is_the_same(seed):
    """Parallel arcs merged into one transition with the summed weight give
    Valmari the same lumping (the form used when the reader would refuse more
    transitions than states squared)."""
    import subprocess
    off, idx = _messy(seed)
    wt = np.random.default_rng(seed).integers(1, 6, size=len(idx)).astype(np.uint64) if seed % 2 else None
    labels = []
    for merge in (False, True):
        txt = subprocess.run([oracle.REF_VALMARI], input=oracle.mdp_text(off, idx, wt, None, merge=merge),
                             capture_output=True, check=True, timeout=120).stdout.decode()
        labels.append(oracle._canon_u64(oracle._parse_ref_output(txt)[4]))
    assert np.array_equal(labels[0], labels[1])
