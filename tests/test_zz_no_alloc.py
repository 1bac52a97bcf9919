"""The allocation-free entry point (rbsc_refine_noalloc) against the regular
one (rbsc_refine), through the C ABI.

rbsc_refine_noalloc exists for callers that cannot allocate device memory
(another framework owns the memory pool, a real-time path must not take the
synchronisation an allocation can bring, or the host only hands out pointers
into memory it manages).  It keeps all its scratch in one static device array
shared by every call, so this test checks two calls in a row -- the second
must not see anything left over by the first -- and that graphs over the
stated limit are refused.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import _lib, graphs as G

pytestmark = pytest.mark.gpu


def _noalloc(off, idx, wt=None, init=None, opts=None):
    import torch
    lib = _lib.load()
    n = len(off) - 1
    d_off = torch.as_tensor(np.asarray(off, dtype=np.int64), device="cuda")
    d_idx = torch.as_tensor(np.asarray(idx, dtype=np.int32), device="cuda") if len(idx) else None
    d_wt = torch.as_tensor(np.asarray(wt, dtype=np.int64), device="cuda") if wt is not None else None
    d_init = torch.as_tensor(np.asarray(init, dtype=np.int32), device="cuda") if init is not None else None
    d_out = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    d_res = torch.zeros(4, dtype=torch.int32, device="cuda")
    c = _lib.Csr()
    c.n, c.m, c.offsets, c.offset_bytes = n, int(off[-1]), d_off.data_ptr(), 8
    c.indices = d_idx.data_ptr() if d_idx is not None else None
    c.weights = d_wt.data_ptr() if d_wt is not None else None
    torch.cuda.synchronize()
    st = lib.rbsc_refine_noalloc(ctypes.byref(c), d_init.data_ptr() if d_init is not None else None,
                                 d_out.data_ptr(), d_res.data_ptr(), opts, None)
    torch.cuda.synchronize()
    res = d_res.cpu().numpy().view(np.uint32)
    return st, d_out.cpu().numpy().view(np.uint32)[:n], dict(blocks=int(res[0]), rounds=int(res[1]),
                                                                repairs=int(res[2]), status=int(np.int32(res[3])))


def _cases():
    yield "er", *G.er_directed(3000, 12000, seed=5), None, None
    off, idx = G.random_lift(256, 2048, 32, seed=2)          # 8192 nodes, 65536 arcs
    yield "lift", off, idx, None, None
    off, idx = G.rmat(13, 8, seed=7)                           # 8192 nodes
    yield "rmat_degree_colours", off, idx, None, R.degree_bucket_colors(off)
    off, idx = G.er_directed(500, 3000, seed=9)
    wt = np.random.default_rng(9).integers(1, 4, size=len(idx)).astype(np.uint64)
    yield "weighted", off, idx, wt, None
    off, idx = G.complete_bipartite(60, 70)                    # rows longer than a warp
    yield "bipartite", off, idx, None, None


@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_noalloc_matches_refine_twice(case):
    _, off, idx, wt, init = case
    with R.Context(0) as ctx:
        ref = ctx.refine(off, idx, wt, init)
    # another graph first, so the scratch holds a different graph's state
    o2, i2 = G.er_directed(1000, 4000, seed=123)
    _noalloc(o2, i2)
    for _ in range(2):
        st, labels, res = _noalloc(off, idx, wt, init)
        assert st == 0 and res["status"] == 0
        assert np.array_equal(labels, ref.labels)
        assert res["blocks"] == ref.blocks and res["rounds"] == ref.rounds


def test_noalloc_rejects_graphs_over_the_limit():
    n = _lib.NOALLOC_MAX_NODES + 1
    off, idx = G.cycle(n)
    st, _, _ = _noalloc(off, idx)
    assert st == -7  # RBSC_ERR_TOO_LARGE
    assert b"exceeds the limit" in _lib.load().rbsc_last_error(None)


def test_noalloc_exact_under_forced_collisions():
    off, idx = G.er_directed(800, 3000, seed=4)
    with R.Context(0) as ctx:
        ref = ctx.refine(off, idx)
    o = _lib.Opts()
    _lib.load().rbsc_opts_default(ctypes.byref(o))
    o.test_hash_bits = -1  # no signatures: every split comes from the exact check
    st, labels, res = _noalloc(off, idx, opts=ctypes.byref(o))
    assert st == 0 and res["status"] == 0 and res["repairs"] > 0
    assert np.array_equal(labels, ref.labels) and res["blocks"] == ref.blocks
