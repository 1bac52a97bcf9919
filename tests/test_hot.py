"""Hot heads of the first signature pass: the class ranks of the most
pointed-to nodes are read from shared memory (k_signature_hot).  The
partition, the canonical labels and the round count must equal the plain
kernel's and the oracle's, whichever nodes are hot."""
import numpy as np
import pytest

import rbsc_b200 as R
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat18():
    off, idx = R.gen_rmat_host(18, 20, seed=6)
    assert len(idx) >= (1 << 22)  # hot heads apply from 2^22 arcs
    return off, idx


def _resident(off, idx, wt, init, **opts):
    """Two refinements of one resident graph (the first builds the hot heads,
    the second reuses them)."""
    with R.Context(0, **opts) as ctx:
        g = ctx.upload(off, idx, wt)
        r1 = g.refine(init)
        r2 = g.refine(init)
        g.free()
    return r1, r2


def _same(r, ex):
    assert r.done == 1 and r.verified == 1
    assert r.blocks == ex.blocks and r.rounds == ex.rounds
    assert np.array_equal(r.labels, ex.labels)


@pytest.mark.parametrize("weighted", [False, True], ids=["unweighted", "weighted"])
def test_hot_heads_equal_the_oracle(rmat18, weighted):
    off, idx = rmat18
    wt = np.random.default_rng(3).integers(1, 4, len(idx), dtype=np.uint64) if weighted else None
    init = R.degree_bucket_colors(off)
    ex = oracle.refine_exact(off, idx, wt, init)
    h1, h2 = _resident(off, idx, wt, init)
    p1, _ = _resident(off, idx, wt, init, sig_kernel=1)
    assert 0 < h1.first_signature_hot <= (1 << 17)
    assert h2.first_signature_hot == h1.first_signature_hot
    assert p1.first_signature_hot == 0
    for r in (h1, h2, p1):
        _same(r, ex)


@pytest.mark.parametrize("weighted", [False, True], ids=["unweighted", "weighted"])
def test_hot_heads_by_tensor_copies_equal_the_oracle(rmat18, weighted):
    """sig_kernel 4: each warp's tile of heads is brought into shared memory
    by the tensor memory accelerator (128-byte swizzled boxes); the last tile
    is partial (the arc count is not a multiple of 512)."""
    off, idx = rmat18
    assert len(idx) % 512 != 0
    wt = np.random.default_rng(5).integers(1, 4, len(idx), dtype=np.uint64) if weighted else None
    init = R.degree_bucket_colors(off)
    ex = oracle.refine_exact(off, idx, wt, init)
    t1, t2 = _resident(off, idx, wt, init, sig_kernel=4)
    assert 0 < t1.first_signature_hot <= (1 << 17)
    for r in (t1, t2):
        _same(r, ex)


@pytest.mark.parametrize("sig_kernel", [3, 4])
@pytest.mark.parametrize("hot_log2", [10, 13, 17])
def test_hot_table_sizes(rmat18, hot_log2, sig_kernel):
    off, idx = rmat18
    init = R.degree_bucket_colors(off)
    h, _ = _resident(off, idx, None, init, sig_kernel=sig_kernel, hot_log2=hot_log2)
    p, _ = _resident(off, idx, None, init, sig_kernel=1)
    assert 0 < h.first_signature_hot <= (1 << hot_log2)
    assert np.array_equal(h.labels, p.labels) and h.rounds == p.rounds and h.blocks == p.blocks


def test_hot_heads_only_where_they_apply(rmat18):
    off, idx = rmat18
    init = R.degree_bucket_colors(off)
    with R.Context(0) as ctx:
        g = ctx.upload(off, idx)
        # one initial class: the first pass gathers nothing
        assert g.refine(None).first_signature_hot == 0
        # more than 256 classes: 2-byte ranks, plain kernel
        many = (np.arange(len(off) - 1) % 1000).astype(np.uint32)
        r = g.refine(many)
        assert r.first_signature_hot == 0
        _same(r, oracle.refine_exact(off, idx, None, many))
        assert g.refine(init).first_signature_hot > 0
        # the staged kernel when asked for
        ctx.set_opts(sig_kernel=2)
        assert g.refine(init).first_signature_hot == 0
        g.free()
        ctx.set_opts(sig_kernel=0)
        # a one-shot call keeps no second copy of the heads
        assert ctx.refine(off, idx, init=init).first_signature_hot == 0
        # below 2^22 arcs
        soff, sidx = R.gen_rmat_host(14, 16, seed=2)
        gs = ctx.upload(soff, sidx)
        assert gs.refine(R.degree_bucket_colors(soff)).first_signature_hot == 0
        gs.free()


def test_no_hot_heads_without_skew():
    """Every node has in-degree 20 (a circulant graph): no threshold admits at
    most 2^17 nodes, so the plain kernel runs, with the same result.  N is a
    multiple of the marking's period 7, so the partition is stable at once
    (a period that does not divide N would take ~N/40 rounds to resolve)."""
    n, d = 7 << 15, 20
    off = np.arange(n + 1, dtype=np.uint64) * d
    idx = ((np.arange(n, dtype=np.uint64)[:, None] + np.arange(1, d + 1, dtype=np.uint64)[None, :]) % n)
    idx = np.sort(idx, axis=1).astype(np.uint32).ravel()
    init = (np.arange(n) % 7 == 0).astype(np.uint32)
    h, _ = _resident(off, idx, None, init)
    assert h.first_signature_hot == 0
    _same(h, oracle.refine_exact(off, idx, None, init))
