"""The multi-GPU path of bench.py: N independent replicas (the refinement
does not shard), one process per GPU, the job timed by the slowest rank.
Its host logic runs here as two `gloo` ranks on the CPU: the max-over-ranks
reduction and the whole-job value."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's own times; the job takes the slowest rank's
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.5], dist)
        v = bench.replica_value(world, 1000, 5, 4, got[0])
        q.put((rank, got, v))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, got, v in res:
        assert got == [2.0, 10.0, 3.5]
        assert v == pytest.approx(2 * 1000 * 5 * 4 / 0.002)


def test_single_process_is_the_identity():
    assert bench.max_over_ranks([1.5, 2.5], None) == [1.5, 2.5]
    assert bench.replica_value(1, 263429291, 5, 20, 80.0) == pytest.approx(263429291 * 5 * 20 / 0.08)
