"""The pass kernels' knobs (hand-off threshold to the persistent kernel,
blocks per SM) and the autotuner that picks them (rbsc_graph_autotune).
Every setting must give the same partition; the tuner must choose a setting
whose result equals the default's."""
import ctypes

import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import _lib, graphs as G
from oracle import oracle


def test_opts_layout_unchanged():
    # the two knobs took two of the reserved words: the struct keeps its size
    assert ctypes.sizeof(_lib.Opts) == 4 * 4 + 8 + 4 * 2 + 4 * 6
    lib = _lib.load()
    o = _lib.Opts()
    lib.rbsc_opts_default(ctypes.byref(o))
    assert o.persist_log2 == 0 and o.grid_per_sm == 0
    sp = _lib.TuneSpace()
    lib.rbsc_tune_space_default(ctypes.byref(sp))
    assert sp.n_persist >= 2 and sp.n_grid >= 2 and sp.reps >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("sig_kernel", [1, 2])
@pytest.mark.parametrize("persist_log2,grid", [(-1, 4), (10, 8), (16, 32), (31, 2)])
def test_knobs_keep_the_partition(persist_log2, grid, sig_kernel):
    off, idx = G.rmat(12, 8, seed=4)
    init = R.degree_bucket_colors(off)
    ex = oracle.refine_exact(off, idx, init=init)
    with R.Context(0, persistent=persist_log2 >= 0, persist_log2=persist_log2, grid_per_sm=grid,
                   sig_kernel=sig_kernel) as ctx:
        g = ctx.upload(off, idx)
        for _ in range(2):
            r = g.refine(init)
            assert r.blocks == ex.blocks and r.rounds == ex.rounds and np.array_equal(r.labels, ex.labels)
        g.free()


@pytest.mark.gpu
def test_autotune_chooses_an_equivalent_setting():
    off, idx, gn, lab = R.gen_wl_batch(2000, 10, 200, 8, seed=3)
    import torch
    d_init = torch.from_numpy(lab.view(np.int32)).cuda()
    with R.Context(0) as ctx:
        g = ctx.upload(off, idx)
        ref = g.refine(lab)
        t = g.autotune(d_init.data_ptr(), persist_log2=[14, 22, -1], grid_per_sm=[4, 16], use_graph=[1, 0],
                       sig_kernel=[1, 2], reps=2)
        assert t["candidates"] == 24 and t["failed"] == 0
        assert t["best_ms"] <= t["default_ms"] + 1e-9
        assert len(t["table"]) == 24
        r = g.refine(lab)  # under the chosen setting
        assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)
        g.free()
