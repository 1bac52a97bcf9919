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
from oracle import oracle
from rbsc_b200 import _lib, graphs as G

pytestmark = pytest.mark.gpu


def _noalloc(off, idx, wt=None, init=None, opts=None, offset_bytes=8, m=None):
    import torch
    lib = _lib.load()
    n = len(off) - 1
    odt = np.int64 if offset_bytes == 8 else np.int32
    d_off = torch.as_tensor(np.asarray(off, dtype=np.int64).astype(odt), device="cuda")
    d_idx = torch.as_tensor(np.asarray(idx, dtype=np.uint32).view(np.int32), device="cuda") if len(idx) else None
    d_wt = torch.as_tensor(np.asarray(wt, dtype=np.int64), device="cuda") if wt is not None else None
    d_init = torch.as_tensor(np.asarray(init, dtype=np.int32), device="cuda") if init is not None else None
    d_out = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    d_res = torch.zeros(4, dtype=torch.int32, device="cuda")
    c = _lib.Csr()
    c.n, c.m, c.offsets, c.offset_bytes = n, int(off[-1]) if m is None else m, d_off.data_ptr(), offset_bytes
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


@pytest.mark.parametrize("offset_bytes", [8, 4])
@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_noalloc_matches_refine_twice(case, offset_bytes):
    _, off, idx, wt, init = case
    with R.Context(0) as ctx:
        ref = ctx.refine(off, idx, wt, init)
    ex = oracle.refine_exact(off, idx, wt, init)
    assert np.array_equal(ref.labels, ex.labels) and ref.blocks == ex.blocks and ref.rounds == ex.rounds
    # another graph first, so the scratch holds a different graph's state
    o2, i2 = G.er_directed(1000, 4000, seed=123)
    _noalloc(o2, i2)
    for _ in range(2):
        st, labels, res = _noalloc(off, idx, wt, init, offset_bytes=offset_bytes)
        assert st == 0 and res["status"] == 0
        assert np.array_equal(labels, ref.labels)
        assert res["blocks"] == ref.blocks and res["rounds"] == ref.rounds


def test_noalloc_empty_graph():
    st, labels, res = _noalloc(np.zeros(1, dtype=np.int64), np.zeros(0, dtype=np.uint32))
    assert st == 0 and res == dict(blocks=0, rounds=0, repairs=0, status=0) and labels.size == 0


def test_noalloc_not_converged_within_max_rounds():
    off, idx = G.path(40)  # needs about 40 rounds
    o = _lib.Opts()
    _lib.load().rbsc_opts_default(ctypes.byref(o))
    o.max_rounds = 1
    st, _, res = _noalloc(off, idx, opts=ctypes.byref(o))
    assert st == 0 and res["status"] == -4  # RBSC_ERR_NOT_CONVERGED
    # and the same call without the limit still matches the oracle afterwards
    st, labels, res = _noalloc(off, idx)
    ex = oracle.refine_exact(off, idx)
    assert st == 0 and res["status"] == 0 and np.array_equal(labels, ex.labels) and res["rounds"] == ex.rounds


def _malformed():
    off, idx = G.er_directed(300, 1200, seed=8)
    off = np.asarray(off, dtype=np.int64)
    idx = np.asarray(idx, dtype=np.uint32)
    bad = idx.copy()
    bad[len(bad) // 2] = 300                              # head == N
    yield "head_eq_n", off, bad, None
    bad = idx.copy()
    bad[-1] = 0xFFFFFFF0                                   # head far outside any array
    yield "head_huge", off, bad, None
    o = off.copy()
    o[150] = o[151] + 5                                    # offsets decreasing
    yield "offsets_decreasing", o, idx, None
    o = off.copy()
    o[0] = 3                                               # offsets[0] != 0
    yield "offsets_first", o, idx, None
    yield "offsets_last_ne_m", off, idx, len(idx) - 7      # offsets[N] != M


@pytest.mark.parametrize("case", list(_malformed()), ids=lambda c: c[0])
def test_noalloc_rejects_malformed_graph_on_the_device(case):
    _, off, idx, m = case
    st, labels, res = _noalloc(off, idx, m=m)
    assert st == 0 and res["status"] == -1  # RBSC_ERR_INVALID, found by the kernel's own check
    assert np.all(labels == 0xFFFFFFFF)     # the output is left untouched
    # the next call on a good graph is unaffected
    o2, i2 = G.er_directed(300, 1200, seed=8)
    st, labels, res = _noalloc(o2, i2)
    assert st == 0 and res["status"] == 0 and np.array_equal(labels, oracle.refine_exact(o2, i2).labels)


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
