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


# --------------------------------------------------------------------------
# One scene split across ranks by slabs of the screen (math_b200/tiles.py),
# with the reference painter (the oracle) rendering each slab.


def test_slab_rows_cover_the_screen_once():
    from math_b200 import tiles

    for rows in (1, 2, 7, 64, 96):
        for world in range(1, min(rows, 9) + 1):
            slabs = [tiles.slab_rows(rows, r, world) for r in range(world)]
            assert slabs[0][0] == 0 and slabs[-1][1] == rows
            assert all(a[1] == b[0] for a, b in zip(slabs, slabs[1:]))
            sizes = [e - b for b, e in slabs]
            assert max(sizes) - min(sizes) <= 1
            for b, e in slabs:
                sb, se = tiles.source_rows(rows, b, e)
                assert sb == max(0, b - 1) and se == min(rows, e + 1)
    with pytest.raises(ValueError):
        tiles.slab_rows(3, 0, 4)


def tile_rank(rank: int, world: int, port: int, out):
    import sys

    sys.path.insert(0, str(ROOT))
    import numpy as np

    from math_b200 import scenes, tiles
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        desc = scenes.cornell_3d(size=(12, 10), subdivisions=2)
        s = oracle.Scene(desc, "double", False)
        size = desc["projector"]["size"]
        rows = size[-1]
        b, e = tiles.slab_rows(rows, rank, world)
        sb, se = tiles.source_rows(rows, b, e)
        # the slab's paths and those of its halo rows, accumulated; only the
        # slab's own pixels are complete
        first, last = tiles.pixel_range(size, sb, se)
        rgb, _ = s.render_image_range(16, 5, 1, first, last, threads=2)
        lo, hi = tiles.pixel_range(size, b, e)
        whole = tiles.gather_image(np.ascontiguousarray(rgb[lo:hi]), rank, world, rows, size)
        if rank == 0:
            out["image"] = whole
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world", [2, 3])
def test_slabs_rendered_on_ranks_make_the_whole_image(oracle_lib, world):
    """Each gloo rank renders its slab with the reference painter (per-pixel
    seeded streams, the halo rows recomputed); rank 0 gathers the slabs and
    the result equals the one-rank image bit for bit."""
    from math_b200 import scenes

    port = free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(tile_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    desc = scenes.cornell_3d(size=(12, 10), subdivisions=2)
    ref, _ = oracle_lib.Scene(desc, "double", False).render_image(16, 5, 1, threads=2)
    import numpy as np

    assert np.array_equal(out["image"], ref)
