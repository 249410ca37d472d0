"""bench.py's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1), each
with a different device time; the job time is the max over ranks and the
throughput counts every rank's work.  Replicas exchange nothing else."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_seconds = 1.0 + rank  # rank 1 is the slow one
        bench.barrier(world)
        tmax = bench.max_over_ranks(my_seconds, world)
        total = bench.sum_over_ranks(10.0 * (rank + 1), world)
        rate = bench.aggregate_rate(1000.0, world, tmax)
        q.put((rank, tmax, total, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_aggregate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, tmax, total, rate in res:
        assert tmax == 2.0
        assert total == 30.0
        assert rate == pytest.approx(1000.0 * 2 / 2.0)


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.aggregate_rate(100.0, 1, 2.0) == 50.0
