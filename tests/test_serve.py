"""Serving (rbsc_serve_*): admission by device footprint, packing of small
jobs, arrival order, queue limits and shutdown.

These run on the CPU: the server's test hook `dry_run` replaces every
refinement by a host sleep of a fixed time per arc, so the scheduling and
accounting code runs unchanged without a GPU.  The GPU tests of the same
server (results alone vs in the mix) are in test_serve_gpu.py."""
import threading
import time

import numpy as np
import pytest

import rbsc_b200 as R
from rbsc_b200._lib import RbscError


@pytest.fixture(scope="module")
def er2k():
    return R.gen_er_host(2000, 4.0, seed=11)


def test_footprint_grows_with_size():
    a = R.serve_footprint(1000, 4000)
    b = R.serve_footprint(2000, 8000)
    assert 0 < a < b
    assert R.serve_footprint(1000, 4000, weighted=True) > a
    assert R.serve_footprint(1000, 4000, graphs=10) > a


def test_admission_stays_within_budget(er2k):
    off, idx = er2k
    fp = R.serve_footprint(len(off) - 1, len(idx))
    budget = int(fp * 2.5)  # room for two jobs at a time
    with R.Server(slots=4, hbm_budget=budget, pack_max_graphs=1, dry_run_ns_per_arc=300) as srv:
        ids = [srv.submit(off, idx) for _ in range(12)]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r.status == 0 and r.packed == 1 for r in res)
    assert st["completed"] == 12 and st["failed"] == 0
    assert st["peak_reserved"] <= budget
    assert st["peak_busy_slots"] == 2
    assert st["reserved"] == 0 and st["running"] == 0 and st["queued"] == 0


def test_jobs_start_in_arrival_order(er2k):
    off, idx = er2k
    with R.Server(slots=1, pack_max_graphs=1, dry_run_ns_per_arc=200) as srv:
        t_sub, ids = [], []
        for _ in range(8):
            t_sub.append(time.perf_counter() * 1e3)
            ids.append(srv.submit(off, idx))
        res = [srv.wait(i) for i in ids]
    starts = [t + r.queue_ms for t, r in zip(t_sub, res)]
    for a, b, ra in zip(starts, starts[1:], res):
        assert b >= a + ra.service_ms - 0.5


def test_small_jobs_are_packed():
    off, idx = R.gen_er_host(200, 3.0, seed=5)
    m = len(idx)
    with R.Server(slots=2, pack_max_arcs=1 << 12, pack_max_graphs=8, pack_arc_budget=5 * m,
                  dry_run_ns_per_arc=2000) as srv:
        ids = [srv.submit(off, idx) for _ in range(120)]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r.status == 0 for r in res)
    packs = [r.packed for r in res]
    assert max(packs) > 1
    assert max(packs) <= 5                      # arc budget: 5 jobs of m arcs
    assert st["packed_jobs"] == sum(1 for p in packs if p > 1)
    assert abs(sum(1.0 / p for p in packs) - st["batches"]) < 1e-6  # each pack of k counted k times


def test_large_jobs_are_not_packed(er2k):
    off, idx = er2k
    small_off, small_idx = R.gen_er_host(50, 2.0, seed=2)
    with R.Server(slots=1, pack_max_arcs=len(small_idx), dry_run_ns_per_arc=100) as srv:
        ids = []
        for k in range(20):
            ids.append(srv.submit(off, idx) if k % 4 == 0 else srv.submit(small_off, small_idx))
        res = [srv.wait(i) for i in ids]
    for k, r in enumerate(res):
        if k % 4 == 0:
            assert r.packed == 1


def test_small_jobs_do_not_wait_behind_a_burst_of_large_ones():
    """With every executor but one running a large job, the last one goes to
    the small jobs that wait, before the next large job (which still starts
    as soon as they leave it free).  Two executors: a short large job, a long
    large job, then a third large job and three small ones."""
    short_l = R.gen_er_host(1000, 4.0, seed=21)
    long_l = R.gen_er_host(10000, 4.0, seed=22)
    big = R.gen_er_host(2000, 4.0, seed=23)
    tiny = R.gen_er_host(30, 2.0, seed=24)
    with R.Server(slots=2, pack_max_arcs=1 << 10, pack_max_graphs=8, dry_run_ns_per_arc=2000) as srv:
        t_sub, ids = [], []
        for off, idx in (short_l, long_l, big, tiny, tiny, tiny):
            t_sub.append(time.perf_counter() * 1e3)
            ids.append(srv.submit(off, idx))
        res = [srv.wait(i) for i in ids]
    assert all(r.status == 0 for r in res)
    start = [t + r.queue_ms for t, r in zip(t_sub, res)]
    assert res[2].packed == 1 and all(r.packed >= 1 for r in res[3:])
    # the small jobs started before the third large job, which did not wait
    # for the long one to finish
    assert max(start[3:]) < start[2]
    assert start[2] < start[1] + res[1].service_ms


def test_weighted_jobs_run_alone():
    off, idx = R.gen_er_host(60, 2.0, seed=3)
    wt = np.ones(len(idx), dtype=np.uint64)
    with R.Server(slots=1, dry_run_ns_per_arc=5000) as srv:
        ids = [srv.submit(off, idx, wt=wt) for _ in range(6)]
        assert all(srv.wait(i).packed == 1 for i in ids)


def test_errors_and_limits(er2k):
    off, idx = er2k
    fp = R.serve_footprint(len(off) - 1, len(idx))
    with R.Server(slots=1, hbm_budget=fp // 2, dry_run_ns_per_arc=1) as srv:
        with pytest.raises(RbscError) as e:
            srv.submit(off, idx)
        assert e.value.status == -7
        assert srv.stats()["rejected"] == 1
    with R.Server(slots=1, queue_cap=2, pack_max_graphs=1, dry_run_ns_per_arc=5000) as srv:
        first = srv.submit(off, idx)          # starts at once
        time.sleep(0.01)
        a, b = srv.submit(off, idx), srv.submit(off, idx)
        with pytest.raises(RbscError) as e:
            srv.submit(off, idx)
        assert e.value.status == -8
        assert srv.poll(b) is None            # still pending
        for j in (first, a, b):
            assert srv.wait(j).status == 0
        with pytest.raises(RbscError) as e:
            srv.wait(first)                   # a result is handed out once
        assert e.value.status == -1
        with pytest.raises(RbscError):
            srv.poll(123456)


def test_wait_with_timeout(er2k):
    off, idx = er2k
    with R.Server(slots=1, dry_run_ns_per_arc=20000) as srv:   # ~160 ms per job
        j = srv.submit(off, idx)
        assert srv.wait(j, timeout_ms=1) is None
        assert srv.wait(j).status == 0


def test_shutdown_cancels_waiting_jobs(er2k):
    off, idx = er2k
    srv = R.Server(slots=1, pack_max_graphs=1, dry_run_ns_per_arc=2500)  # ~20 ms per job
    for _ in range(50):
        srv.submit(off, idx)
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 < 0.5     # only the running job is finished


def test_concurrent_submitters():
    graphs = [R.gen_er_host(100 + 37 * k, 3.0, seed=k) for k in range(4)]
    errors = []
    with R.Server(slots=3, pack_max_arcs=1 << 10, dry_run_ns_per_arc=500) as srv:
        def worker(k):
            try:
                off, idx = graphs[k]
                ids = [srv.submit(off, idx) for _ in range(40)]
                for i in ids:
                    r = srv.wait(i)
                    assert r.status == 0
            except Exception as ex:  # pragma: no cover - reported below
                errors.append(ex)
        ts = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        st = srv.stats()
    assert not errors
    assert st["completed"] == 160 and st["peak_busy_slots"] <= 3
