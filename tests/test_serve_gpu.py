"""Serving on the GPU: every job's result is the same alone and in the mix.

A mix of graphs of uneven sizes (random lifts, R-MAT, Erdos-Renyi, with and
without initial colours, one weighted) is refined once alone through
rbsc_refine and once through a server that runs them concurrently on several
slots, packs the small ones into batch refinements and admits by device
footprint.  Integer work, so the tolerance is zero: canonical labels and block
counts must be identical (round counts too for jobs that ran alone)."""
import time

import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200 import graphs as G
from oracle import oracle

pytestmark = pytest.mark.gpu


def _mix():
    jobs = []
    rng = np.random.default_rng(7)
    for k in range(36):
        kind = k % 4
        if kind == 0:
            off, idx = R.gen_lift_host(int(rng.integers(16, 400)), 3.0, int(rng.integers(2, 17)), seed=100 + k)
        elif kind == 1:
            off, idx = G.rmat(int(rng.integers(6, 13)), int(rng.integers(2, 9)), seed=200 + k)
        elif kind == 2:
            off, idx = R.gen_er_host(int(rng.integers(20, 3000)), float(rng.uniform(1.0, 6.0)), seed=300 + k)
        else:
            off, idx = G.random_lift(64, 256, 8, seed=400 + k)
        init = None
        if k % 3 == 1:
            init = rng.integers(1, 5, size=len(off) - 1, dtype=np.uint32)
        elif k % 3 == 2:
            init = R.degree_bucket_colors(off)
        jobs.append((off, idx, None, init))
    # a larger job, a weighted one and a one-node graph
    jobs.append(R.gen_lift_host(4096, 8.0, 32, seed=5) + (None, None))
    off, idx = R.gen_er_host(500, 4.0, seed=9)
    jobs.append((off, idx, rng.integers(1, 4, size=len(idx), dtype=np.uint64), None))
    jobs.append((np.array([0, 0], dtype=np.uint64), np.zeros(0, dtype=np.uint32), None, None))
    return jobs


@pytest.fixture(scope="module")
def mix():
    jobs = _mix()
    alone = []
    with R.Context(0) as ctx:
        for off, idx, wt, init in jobs:
            alone.append(ctx.refine(off, idx, wt, init))
    return jobs, alone


def _check(res, ref):
    assert res.status == 0, res.error
    assert res.blocks == ref.blocks
    assert np.array_equal(res.labels, ref.labels)
    if res.packed == 1:
        assert res.rounds == ref.rounds


def test_alone_matches_oracle(mix):
    """Every job of the mix, refined alone, equals the oracle (labels, blocks
    and rounds), so the in-mix results below are pinned to the oracle too."""
    jobs, alone = mix
    for (off, idx, wt, init), r in zip(jobs, alone):
        ex = oracle.refine_exact(off, idx, wt, init)
        assert r.blocks == ex.blocks and np.array_equal(r.labels, ex.labels)
        assert r.rounds == ex.rounds


def test_mix_equals_alone(mix):
    jobs, alone = mix
    with R.Server(0, slots=3, pack_max_arcs=1 << 14, pack_max_graphs=16) as srv:
        ids = [srv.submit(off, idx, wt, init) for off, idx, wt, init in jobs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for r, a in zip(res, alone):
        _check(r, a)
    assert st["packed_jobs"] > 0            # some jobs ran packed
    assert st["completed"] == len(jobs) and st["failed"] == 0


def test_mix_with_arrivals_while_running(mix):
    """Jobs arrive while others are on the GPU (continuous admission)."""
    jobs, alone = mix
    order = np.random.default_rng(3).permutation(len(jobs))
    with R.Server(0, slots=2, pack_max_arcs=1 << 12) as srv:
        ids = {}
        for k, j in enumerate(order):
            off, idx, wt, init = jobs[j]
            ids[j] = srv.submit(off, idx, wt, init)
            if k % 5 == 4:
                time.sleep(0.002)
        res = {j: srv.wait(i) for j, i in ids.items()}
    for j, r in res.items():
        _check(r, alone[j])


def test_mix_under_tight_budget(mix):
    """A budget that admits about one large job at a time: jobs wait for
    memory, the reserved footprint never exceeds the budget, results stay
    exact."""
    jobs, alone = mix
    big = max(R.serve_footprint(len(o) - 1, len(i), w is not None) for o, i, w, _ in jobs)
    budget = int(big * 1.3)
    with R.Server(0, slots=4, hbm_budget=budget, pack_max_arcs=1 << 13) as srv:
        ids = [srv.submit(off, idx, wt, init) for off, idx, wt, init in jobs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for r, a in zip(res, alone):
        _check(r, a)
    assert st["peak_reserved"] <= budget
