"""Multi-GPU bench aggregation on CPU: two gloo ranks (replicas) agree on the
slowest rank's time and report the whole-job rate from it."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        elapsed = [0.5, 0.8][rank]  # seconds each replica took
        t = bench.max_over_ranks(elapsed, "cpu")
        q.put((rank, t, bench.job_rate(1000.0, world, t)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, t, rate in out:
        assert t == pytest.approx(0.8)
        assert rate == pytest.approx(2 * 1000.0 / 0.8)


def test_job_rate_single():
    assert bench.job_rate(20000 * 256, 1, 0.01) == pytest.approx(5.12e8)
