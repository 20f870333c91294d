"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): each rank
renders a disjoint block of samples of the same frame, and the whole-job
figures are the slowest rank's time with counts summed over ranks. The GPU
side needs no collective (tests/test_gpu_render.py checks that sample blocks
rendered apart combine into the one-render estimate)."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        first, count = bench.sample_block(rank, 64)
        t, rays, h2d = bench.reduce_max_sum(dist, "cpu", 100.0 + 7.0 * rank, 1000 + rank, 5)
        out[rank] = (first, count, t, rays, h2d)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    blocks = sorted((res[r][0], res[r][0] + res[r][1]) for r in range(world))
    assert blocks == [(0, 64), (64, 128)]  # disjoint, contiguous
    for r in range(world):
        assert res[r][2] == pytest.approx(107.0)  # slowest rank
        assert res[r][3] == pytest.approx(2001.0)  # summed rays
        assert res[r][4] == pytest.approx(10.0)


def test_single_process_passthrough():
    assert bench.reduce_max_sum(None, "cpu", 3.0, 4, 5) == (3.0, 4.0, 5.0)
    assert bench.sample_block(0, 16) == (0, 16)
