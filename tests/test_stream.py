"""Graphs whose arcs stay in host memory (rbsc_graph_upload_streamed): the
signature passes stream the arcs in batches through two device buffers; the
compaction brings the active arcs into device memory once they fit the
resident capacity.  The result must be the in-HBM refinement's, bit for bit
(canonical labels, block count, round count), whatever the batch size and the
resident capacity, for pinned and for pageable host arrays."""
import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import graphs as G
from oracle import oracle

pytestmark = pytest.mark.gpu


def _pinned_copy(a):
    import torch
    tdt = {np.dtype(np.uint32): torch.int32, np.dtype(np.uint64): torch.int64}[a.dtype]
    t = torch.empty(max(a.size, 1), dtype=tdt, pin_memory=True)
    v = t.numpy().view(a.dtype)[: a.size]
    v[:] = a
    return v, t


CASES = [
    ("rmat12", lambda: G.rmat(12, 8, seed=3), None),
    ("lift", lambda: G.random_lift(256, 2048, 16, seed=2), None),
    ("er", lambda: G.er_directed(3000, 15000, seed=4), None),
    ("rmat12_degclass", lambda: G.rmat(12, 8, seed=3), "degree"),
    ("lift_labels", lambda: G.random_lift(128, 1024, 8, seed=5), "random"),
]


def _init(kind, off):
    if kind == "degree":
        return R.degree_bucket_colors(off)
    if kind == "random":
        return np.random.default_rng(1).integers(1, 6, size=len(off) - 1).astype(np.uint32)
    return None


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("batch", [512, 3000, 0], ids=["b512", "b3000", "quarter"])
@pytest.mark.parametrize("name,make,init_kind", CASES, ids=[c[0] for c in CASES])
def test_streamed_equals_in_hbm(ctx, name, make, init_kind, batch):
    off, idx = make()
    init = _init(init_kind, off)
    ref = ctx.upload(off, idx).refine(init)
    g = ctx.upload_streamed(off, idx, batch_arcs=batch)
    try:
        r = g.refine(init)
        r2 = g.refine(init)  # repeated refinement of the same streamed graph
    finally:
        g.free()
    for x in (r, r2):
        assert x.blocks == ref.blocks and x.rounds == ref.rounds
        assert np.array_equal(x.labels, ref.labels)
        assert x.streamed_passes >= 1 and x.streamed_bytes >= 4 * len(idx)


def test_streamed_without_compaction(ctx):
    """resident capacity 1 arc: every pass streams the whole arc set."""
    off, idx = G.rmat(11, 8, seed=7)
    g = ctx.upload_streamed(off, idx, batch_arcs=1000, resident_arcs=1)
    r = g.refine(R.degree_bucket_colors(off))
    ref = ctx.upload(off, idx).refine(R.degree_bucket_colors(off))
    g.free()
    assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)
    assert r.streamed_passes == r.rounds
    assert r.streamed_bytes == 4 * len(idx) * r.rounds


def test_streamed_weighted_pinned(ctx):
    off, idx = G.er_directed(800, 6400, seed=9)
    wt = np.random.default_rng(2).integers(1, 4, size=len(idx)).astype(np.uint64)
    idx_p, t1 = _pinned_copy(idx)
    wt_p, t2 = _pinned_copy(wt)
    ex = oracle.refine_exact(off, idx, wt)
    g = ctx.upload_streamed(off, idx_p, wt_p, batch_arcs=700)
    r = g.refine()
    g.free()
    assert r.blocks == ex.blocks and np.array_equal(r.labels, ex.labels) and r.rounds == ex.rounds
    assert r.streamed_bytes >= 12 * len(idx)


def test_streamed_exact_check_repairs(ctx):
    """Signatures dropped entirely on a streamed graph: every split comes from
    the exact check (reading the host arcs) and its repair."""
    off, idx = G.rmat(10, 8, seed=3)
    init = R.degree_bucket_colors(off)
    ex = oracle.refine_exact(off, idx, init=init)
    ctx.set_opts(test_hash_bits=-1)
    try:
        g = ctx.upload_streamed(off, idx, batch_arcs=600)
        r = g.refine(init)
        g.free()
    finally:
        ctx.set_opts(test_hash_bits=0)
    assert r.blocks == ex.blocks and np.array_equal(r.labels, ex.labels)
    assert r.repairs >= 1


def test_streamed_graph_loop_and_host_loop(ctx):
    off, idx = G.rmat(13, 8, seed=11)
    init = R.degree_bucket_colors(off)
    ref = ctx.upload(off, idx).refine(init)
    for use_graph in (False, True):
        ctx.set_opts(use_graph=use_graph)
        try:
            g = ctx.upload_streamed(off, idx, batch_arcs=4096)
            r = g.refine(init)
            g.free()
        finally:
            ctx.set_opts(use_graph=True)
        assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)


def test_pinned_generator_matches_host_generator(ctx):
    """rbsc_gen_rmat_pinned (device, source buckets, page-locked output) gives
    the arcs of rbsc_gen_rmat_host; a streamed refinement of it equals the
    in-HBM one."""
    off, idx = R.gen_rmat_host(14, 16, seed=5)
    pg = ctx.gen_rmat_pinned(14, 16, seed=5)
    try:
        assert pg.n == len(off) - 1 and pg.m == len(idx)
        assert np.array_equal(pg.off, off) and np.array_equal(pg.idx, idx)
        init = R.degree_bucket_colors(off)
        ref = ctx.upload(off, idx).refine(init)
        g = ctx.upload_streamed(pg.off, pg.idx)
        r = g.refine(init)
        g.free()
        assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)
    finally:
        pg.free()


def test_one_shot_upload_overlapped_with_the_first_pass(ctx):
    """rbsc_refine of a large unweighted graph copies the heads in chunks during
    the first pass: same result as the resident graph, with and without
    initial colours (a uniform first pass reads no arc: the upload finishes
    before the kernels that do)."""
    off, idx = R.gen_rmat_host(18, 20, seed=6)
    assert len(idx) >= (1 << 22)
    for init in (R.degree_bucket_colors(off), None):
        ref = ctx.upload(off, idx).refine(init)
        r = ctx.refine(off, idx, init=init)
        assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)


def test_one_shot_upload_from_page_locked_heads(ctx):
    """A page-locked source: every chunk's copy is issued when the graph is
    loaded (before the set-up kernels).  Same result as the resident graph and
    as the oracle, with degree classes, with one initial class (a uniform first
    pass: the upload is awaited whole) and twice in a row (reused buffers)."""
    off, idx = R.gen_rmat_host(18, 20, seed=6)
    assert len(idx) >= (1 << 22)
    poff, toff = _pinned_copy(off)
    pidx, tidx = _pinned_copy(idx)
    for init in (R.degree_bucket_colors(off), None, R.degree_bucket_colors(off)):
        ref = ctx.upload(off, idx).refine(init)
        r = ctx.refine(poff, pidx, init=init)
        assert r.blocks == ref.blocks and r.rounds == ref.rounds and np.array_equal(r.labels, ref.labels)
    ex = oracle.refine_exact(off, idx, init=R.degree_bucket_colors(off))
    assert r.blocks == ex.blocks and r.rounds == ex.rounds and np.array_equal(r.labels, ex.labels)
    del toff, tidx


def test_one_shot_upload_from_page_locked_heads_rejects_a_bad_head(ctx):
    off, idx = R.gen_rmat_host(18, 20, seed=7)
    pidx, tidx = _pinned_copy(idx)
    pidx[len(pidx) * 3 // 4] = len(off) - 1 + 5  # a head >= N in the seventh chunk
    for init in (R.degree_bucket_colors(off), None):
        with pytest.raises(R.RbscError) as e:
            ctx.refine(off, pidx, init=init)
        assert e.value.status == -1
    pidx[len(pidx) * 3 // 4] = idx[len(idx) * 3 // 4]
    r = ctx.refine(off, pidx)  # the context is still usable
    assert r.done == 1
    del tidx


def test_one_shot_upload_rejects_a_bad_head(ctx):
    off, idx = R.gen_rmat_host(18, 20, seed=7)
    bad = idx.copy()
    bad[len(bad) * 3 // 4] = len(off) - 1 + 5  # a head >= N in the fourth chunk
    with pytest.raises(R.RbscError) as e:
        ctx.refine(off, bad, init=R.degree_bucket_colors(off))
    assert e.value.status == -1
    r = ctx.refine(off, idx)  # the context is still usable
    assert r.done == 1
