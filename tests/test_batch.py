"""Batches of small graphs refined together in one colour namespace.

CPU: the seeded batch generator (determinism, degrees, symmetry, simple
graphs).  GPU: the batch refinement against the oracle run on the disjoint
union, each graph's own partition against a refinement of that graph alone,
and 1-WL distinguishability (histogram inequality) against refinements of
graph pairs."""
import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import graphs as G
from oracle import oracle


def _graph(off, idx, gn, g):
    a, b = int(gn[g]), int(gn[g + 1])
    o = off[a: b + 1].astype(np.int64)
    sub_idx = idx[o[0]: o[-1]].astype(np.int64) - a
    return (o - o[0]).astype(np.uint64), sub_idx.astype(np.uint32)


def test_generator_rules():
    off, idx, gn, lab = R.gen_wl_batch(300, 10, 120, 8, seed=11)
    off2, idx2, gn2, lab2 = R.gen_wl_batch(300, 10, 120, 8, seed=11, threads=1)
    assert np.array_equal(off, off2) and np.array_equal(idx, idx2) and np.array_equal(gn, gn2) and np.array_equal(lab, lab2)
    assert gn[0] == 0 and gn[-1] == len(off) - 1 and np.all(np.diff(gn.astype(np.int64)) > 0)
    assert lab.min() >= 1 and lab.max() <= 8
    degs = []
    for g in range(300):
        o, ix = _graph(off, idx, gn, g)
        n = len(o) - 1
        assert 4 <= n <= 120
        src = np.repeat(np.arange(n), np.diff(o.astype(np.int64)))
        assert np.all(ix < n) and not np.any(src == ix)  # no loop
        pairs = set(zip(src.tolist(), ix.tolist()))
        assert len(pairs) == len(ix)  # no repeated arc
        assert all((v, u) in pairs for u, v in pairs)  # symmetric
        d = np.diff(o.astype(np.int64))
        if g % 2 == 1:
            assert n % 2 == 0 and np.all(d == 3)
        else:
            degs.append(d.mean())
    assert 3.0 < np.mean(degs) < 5.0
    # a different seed gives a different batch
    off3, idx3, _, _ = R.gen_wl_batch(300, 10, 120, 8, seed=12)
    assert len(idx3) != len(idx) or not np.array_equal(idx3, idx)


def test_generator_rejects_bad_arguments():
    with pytest.raises(R.RbscError):
        R.gen_wl_batch(0)
    with pytest.raises(R.RbscError):
        R.gen_wl_batch(10, 20, 10)


def _hist_from_colors(colors, gn, g):
    c = colors[int(gn[g]): int(gn[g + 1])]
    u, cnt = np.unique(c, return_counts=True)
    return u.astype(np.uint32), cnt.astype(np.uint32)


@pytest.mark.gpu
def test_batch_matches_union_oracle_and_single_graphs():
    off, idx, gn, lab = R.gen_wl_batch(400, 10, 80, 8, seed=3)
    ex = oracle.refine_exact(off, idx, init=lab)
    with R.Context(0) as ctx:
        b = ctx.batch_refine(off, idx, gn, lab)
        assert b.stats.verified == 1 and b.stats.blocks == ex.blocks and b.stats.rounds == ex.rounds
        assert np.array_equal(b.colors, ex.labels)
        assert int(b.hist_offsets[-1]) == len(b.hist_colors)
        for g in range(400):
            hc, hn = _hist_from_colors(ex.labels, gn, g)
            c, k = b.histogram(g)
            assert np.array_equal(c, hc) and np.array_equal(k, hn)
            assert b.blocks[g] == len(hc)
        # each graph's partition is the one a refinement of that graph alone gives
        for g in range(0, 400, 13):
            o, ix = _graph(off, idx, gn, g)
            one = ctx.refine(o, ix, init=lab[int(gn[g]): int(gn[g + 1])])
            assert np.array_equal(one.labels, b.local[int(gn[g]): int(gn[g + 1])])
            assert one.blocks == b.blocks[g]
        # the resident form gives the same
        rg = ctx.upload(off, idx)
        b2 = rg.batch_refine(gn, lab)
        assert np.array_equal(b2.colors, b.colors) and np.array_equal(b2.fingerprint, b.fingerprint)
        rg.free()


@pytest.mark.gpu
def test_wl_distinguishability_is_histogram_inequality():
    """Graph pairs: told apart by refining the pair as a union iff the batch
    gives them different histograms (and fingerprints).  The batch holds
    relabelled copies (same graph, permuted nodes: never told apart) and
    3-regular graphs with one label (1-WL cannot tell same-size ones apart)."""
    rng = np.random.default_rng(7)
    graphs = []
    for i in range(6):
        n = int(rng.integers(12, 40))
        o, ix = G.er_undirected(n, 3.0, seed=100 + i)
        lab = rng.integers(1, 4, size=n).astype(np.uint32)
        graphs.append((o, ix, lab))
        perm = rng.permutation(n)  # relabelled copy
        inv = np.argsort(perm)
        src = np.repeat(np.arange(n), np.diff(o.astype(np.int64)))
        o2, ix2, _ = G.csr_from_arcs(n, perm[src], perm[ix.astype(np.int64)])
        graphs.append((o2, ix2, lab[inv].astype(np.uint32)))
    for i in range(4):
        o, ix = G.random_regular(20, 3, seed=200 + i)
        graphs.append((o, ix, np.ones(20, np.uint32)))
    parts_o, parts_i, parts_l, gn = [], [], [], [0]
    base_n = base_m = 0
    for o, ix, lab in graphs:
        n = len(o) - 1
        parts_o.append(o[:-1].astype(np.uint64) + base_m)
        parts_i.append(ix.astype(np.uint32) + base_n)
        parts_l.append(lab)
        base_n += n
        base_m += len(ix)
        gn.append(base_n)
    off = np.concatenate(parts_o + [np.array([base_m], np.uint64)])
    idx = np.concatenate(parts_i)
    lab = np.concatenate(parts_l)
    gn = np.array(gn, np.uint64)
    with R.Context(0) as ctx:
        b = ctx.batch_refine(off, idx, gn, lab)
        k = len(graphs)
        for i in range(k):
            for j in range(i + 1, k):
                same_hist = all(np.array_equal(x, y) for x, y in zip(b.histogram(i), b.histogram(j)))
                assert same_hist == (b.fingerprint[i] == b.fingerprint[j])
                pair_gn = np.array([0, gn[i + 1] - gn[i], gn[i + 1] - gn[i] + gn[j + 1] - gn[j]], np.uint64)
                oi, ii, li = graphs[i]
                oj, ij, lj = graphs[j]
                po = np.concatenate([oi[:-1].astype(np.uint64), oj.astype(np.uint64) + np.uint64(len(ii))])
                pi = np.concatenate([ii.astype(np.uint32), ij.astype(np.uint32) + np.uint32(len(oi) - 1)])
                ex = oracle.refine_exact(po, pi, init=np.concatenate([li, lj]))
                h_i = _hist_from_colors(ex.labels, pair_gn, 0)
                h_j = _hist_from_colors(ex.labels, pair_gn, 1)
                told_apart = not (np.array_equal(h_i[0], h_j[0]) and np.array_equal(h_i[1], h_j[1]))
                assert told_apart == (not same_hist), (i, j)
        for i in range(0, 12, 2):  # a graph and its relabelled copy
            assert b.fingerprint[i] == b.fingerprint[i + 1]
        assert len(set(b.fingerprint[12:16].tolist())) == 1  # same-size 3-regular, one label


@pytest.mark.gpu
def test_batch_rejects_bad_graph_nodes():
    off, idx, gn, lab = R.gen_wl_batch(20, 10, 30, 8, seed=1)
    with R.Context(0) as ctx:
        bad = gn.copy()
        bad[-1] -= 1
        with pytest.raises(R.RbscError):
            ctx.batch_refine(off, idx, bad, lab)
        bad = gn.copy()
        bad[3] = bad[2]
        with pytest.raises(R.RbscError):
            ctx.batch_refine(off, idx, bad, lab)
