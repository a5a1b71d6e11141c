"""The multi-GPU bookkeeping of bench.py, run as two gloo ranks on CPU: the
timed region is the slowest rank's, and the whole-job throughput counts
every rank's work (weak scaling; the path needs no data-path collective)."""

from __future__ import annotations

import datetime
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out):
    import sys

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    # a rank that never arrives ends the other's collective with an error
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seconds = [1.5, 2.5][rank]
        slowest = bench.slowest_rank(seconds, world, "cpu")
        out[rank] = (slowest, bench.job_throughput(1000.0, world, slowest))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_ranks_take_the_slowest_time_and_count_all_work():
    world = 2
    port = free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for rank in range(world):
        slowest, value = out[rank]
        assert slowest == pytest.approx(2.5)
        assert value == pytest.approx(2 * 1000.0 / 2.5)


def test_one_rank_is_its_own_time():
    import sys

    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.slowest_rank(3.0, 1, "cpu") == 3.0
    assert bench.job_throughput(10.0, 1, 2.0) == 5.0
