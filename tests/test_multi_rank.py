"""Multi-rank host logic on CPU (gloo, world size 2): the whole-job figures of
bench.py are the slowest rank's time with counts summed over ranks; each
rank renders a disjoint set of 64x64 tiles of one frame; and the tile-shard
gather (sundog_b200.shard) assembles the ranks' disjoint films
into the one-GPU frame byte for byte. The GPU side of both decompositions is
tested in tests/test_gpu_render.py."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from sundog_b200 import shard


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
        plan = bench.shard_plan(rank, world, 64)
        t, rays, h2d = bench.reduce_max_sum(dist, "cpu", 100.0 + 7.0 * rank, 1000 + rank, 5)
        out[rank] = (plan, t, rays, h2d)
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
    for r in range(world):
        assert res[r][0] == {"shard_count": 2, "shard_index": r, "spp": 128}
        assert res[r][1] == pytest.approx(107.0)  # slowest rank
        assert res[r][2] == pytest.approx(2001.0)  # summed rays
        assert res[r][3] == pytest.approx(10.0)


def test_single_process_passthrough():
    assert bench.reduce_max_sum(None, "cpu", 3.0, 4, 5) == (3.0, 4.0, 5.0)
    assert bench.shard_plan(0, 1, 16) == {"shard_count": 0, "shard_index": 0, "spp": 16}


def _shard_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        frame = _frame()
        own = torch.from_numpy(shard.owner_map(frame.shape[1], frame.shape[0], world))
        mine = torch.where((own == rank).unsqueeze(-1), frame, torch.zeros_like(frame))
        out[rank] = shard.gather(mine, world).numpy().tobytes()
    finally:
        dist.destroy_process_group()


def _frame():
    g = torch.Generator().manual_seed(7)
    f = torch.randn((130, 200, 4), generator=g)
    f[::7, ::5] = -0.0  # a sum would turn these into +0.0; the gather selects
    return f


def test_tile_shard_gather_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_shard_worker, args=(world, _free_port(), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    want = _frame().numpy().tobytes()
    assert res[0] == want and res[1] == want


def test_owner_map_tiles():
    own = shard.owner_map(200, 130, 5)  # 4 x 3 tiles of 64, edges clipped
    assert own.shape == (130, 200)
    assert own[0, 0] == 0 and own[0, 64] == 1 and own[0, 199] == 3 and own[64, 0] == 4
    assert own[129, 199] == 11 % 5
    counts = [shard.owned_pixels(200, 130, 5, r) for r in range(5)]
    assert sum(counts) == 200 * 130
    assert shard.owned_pixels(200, 130, 16, 13) == 0
    films = [np.where((own == r)[..., None], float(r + 1), 0.0) for r in range(5)]
    assert np.array_equal(shard.assemble(films)[..., 0], own + 1.0)


def test_multi_server_places_jobs_on_least_loaded_device():
    """MultiServer's placement, with stand-in servers (no GPU): each job goes
    to the server with the fewest queued camera paths; finished jobs stop
    counting."""
    from sundog_b200 import abi, serve, workloads

    class FakeJob(object):
        def __init__(self, jid):
            self.id = jid
            self.state = abi.JOB_QUEUED

        def status(self):
            class S(object):
                pass
            st = S()
            st.state = self.state
            return st

    class FakeServer(object):
        def __init__(self):
            self.jobs = []

        def submit(self, scene, base_dir=".", film=True, **opts):
            j = FakeJob(len(self.jobs))
            self.jobs.append(j)
            return j

        def stats(self):
            return len(self.jobs)

        def close(self):
            pass

    assert serve.least_loaded([5, 3, 3, 9]) == 1
    fakes = [FakeServer(), FakeServer(), FakeServer()]
    ms = serve.MultiServer(servers=fakes)
    s = workloads.cornell()
    big = ms.submit(s, width=1024, height=1024, spp=64)    # -> 0
    a = ms.submit(s, width=256, height=256, spp=16)        # -> 1
    b = ms.submit(s, width=256, height=256, spp=16)        # -> 2
    c = ms.submit(s, width=256, height=256, spp=16)        # -> 1 (tie with 2: first)
    assert [big.placement, a.placement, b.placement, c.placement] == [0, 1, 2, 1]
    assert ms.load(0) == 1024 * 1024 * 64
    big.state = abi.JOB_DONE                               # finished: no longer counts
    d = ms.submit(s, width=512, height=512, spp=16)
    assert d.placement == 0 and ms.load(0) == 512 * 512 * 16
    assert ms.stats() == [2, 2, 1]
