"""The multi-rank host logic of bench.py, on CPU: two gloo ranks on
127.0.0.1. On a GPU node each rank drives one GPU and aggregates its own
replica (no collective on the data path); the ranks meet only to time the
job: the job's time is the slowest rank's, and the value counts every
rank's rows."""
import datetime
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        total_ms = 100.0 + 50.0 * rank  # rank 1 is the slower one
        ms, value = bench.weak_scaling(total_ms, 10, 1_000_000, world, None)
        fastest = bench.dist_min(1.0 + rank, world, None)
        bench.dist_barrier(world)
    finally:
        dist.destroy_process_group()
    q.put((rank, ms, value, fastest))


def test_weak_scaling_takes_the_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=180) for _ in procs]
    finally:
        for p in procs:
            p.join(timeout=60)
    assert [p.exitcode for p in procs] == [0, 0]
    assert sorted(r[0] for r in res) == [0, 1]
    for _, ms, value, fastest in res:
        assert ms == pytest.approx(15.0)  # the slower rank's 150 ms over 10 steps
        assert value == pytest.approx(2 * 1_000_000 / 15e-3)  # both ranks' rows
        assert fastest == 1.0


def test_one_rank_needs_no_process_group():
    import bench

    ms, value = bench.weak_scaling(80.0, 8, 4_000_000, 1, None)
    assert ms == pytest.approx(10.0) and value == pytest.approx(4e8)
