"""The multi-rank host logic of bench.py on CPU: two gloo ranks (one process
each, 127.0.0.1 rendezvous) reduce their own timings to the slowest rank's
and compute the same whole-job rate -- what N GPU ranks do over NCCL."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        mine = [1.0 + rank, 10.0 - rank, 3.0]  # each rank's own timings (ms)
        got = bench.max_over_ranks(mine, world)
        rate = bench.job_rate(1 << 30, world, got[0])
        torch.distributed.barrier()
        out.put((rank, got, rate))
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for _, got, rate in res:
        assert got == [2.0, 10.0, 3.0]
        assert rate == pytest.approx((1 << 30) * 2 / 2e-3 / 1e9)


def test_one_rank_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks([4.5, 2.0], 1) == [4.5, 2.0]
    assert bench.job_rate(1 << 30, 1, 1.0) == pytest.approx((1 << 30) / 1e-3 / 1e9)
