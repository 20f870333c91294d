"""The render server (sundog_server_*): continuous batching of tile-passes
from several jobs in one persistent launch.

  * every job's film is the same, bit for bit, alone on the server and
    mixed with other scenes' jobs (ragged edge tiles, spp not a multiple of
    the pass size); with the megakernel engine it is bit-identical to a
    session render of the same scene, size, spp and seed with the megakernel,
    and with the wavefront engine (the default) it equals the wavefront
    session render up to FP32 rounding (the same per-path code compiled into
    other kernels: compared as the engines are in test_gpu_render.py);
  * host-side failures end only the affected job: a missing asset (FAILED
    with the loader's message), a film larger than the device (FAILED, not
    admitted), cancellation of queued and running jobs;
  * one job slot serialises jobs; scene data stays resident between jobs.
"""

import os

import numpy as np
import pytest

from sundog_b200 import abi
from sundog_b200 import scene as sc
from sundog_b200 import serve, workloads
from sundog_b200.scene import scale

pytestmark = pytest.mark.gpu


def session_film(s, base_dir, engine=1, **opts):
    with sc.Session(s, base_dir=base_dir, engine=engine, **opts) as ses:
        ses.render()
        return ses.read()


def close_films(a, b):
    """Films of the same samples from differently compiled kernels: FP32
    rounding, amplified only where a path's decision flips."""
    a = a[..., :3].astype(np.float64)
    b = b[..., :3].astype(np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
    return np.quantile(err, 0.99) <= 1e-4 and np.abs(a.mean() - b.mean()) <= 1e-3 * abs(b.mean())


def mix(asset_dir):
    return [
        (workloads.cornell(), dict(width=96, height=80, spp=12, seed=3)),
        (workloads.instancing(asset_dir), dict(width=136, height=72, spp=5, seed=1)),
        (workloads.volumes(asset_dir), dict(width=100, height=60, spp=6, seed=2)),
        (workloads.cornell(), dict(width=40, height=40, spp=3, seed=9)),
    ]


@pytest.mark.parametrize("engine", [0, 1])
def test_jobs_equal_alone_and_mixed(lib, asset_dir, engine):
    jobs = mix(asset_dir)
    refs = [session_film(s, asset_dir, engine=engine, **o) for s, o in jobs]
    cfg = dict(tile=32, pass_spp=4, iteration_paths=1 << 16, engine=engine)
    # Alone: one job per server.
    alone = []
    for (s, o), ref in zip(jobs, refs):
        with serve.Server(**cfg) as sv:
            film = sv.submit(s, base_dir=asset_dir, **o).wait()
            alone.append(film)
            if engine == 1:
                assert np.array_equal(film, ref)
            else:
                assert close_films(film, ref)
    # Mixed: all jobs in flight together.
    with serve.Server(**cfg) as sv:
        handles = [sv.submit(s, base_dir=asset_dir, **o) for s, o in jobs]
        films = [h.wait() for h in handles]
        st = sv.stats()
    for f, a in zip(films, alone):
        assert np.array_equal(f, a)
    assert st.jobs_done == len(jobs) and st.jobs_failed == 0
    assert st.paths == sum(o["width"] * o["height"] * o["spp"] for _, o in jobs)
    assert st.rays > st.paths and st.iterations > 1
    assert st.scenes_resident == 3  # the two Cornell jobs share one scene


def test_missing_asset_fails_only_that_job(lib, asset_dir, tmp_path):
    bad = sc.Scene()
    bad.render(width=64, height=64, spp=2)
    bad.camera(lookfrom=[0, 1, 5], lookat=[0, 0, 0])
    bad.lambert("grey", color=[0.5, 0.5, 0.5])
    bad.mesh("ghost", "does_not_exist.obj")
    bad.add("mesh:ghost", "grey", scale(1))
    good = workloads.cornell()
    with serve.Server() as sv:
        jb = sv.submit(bad, base_dir=str(tmp_path))
        jg = sv.submit(good, width=48, height=48, spp=2)
        with pytest.raises(serve.JobError, match="does_not_exist.obj"):
            jb.wait()
        assert jb.last.state == abi.JOB_FAILED
        ref = session_film(good, ".", engine=0, width=48, height=48, spp=2)
        assert close_films(jg.wait(), ref)


def test_oversized_job_is_refused(lib):
    with serve.Server() as sv:
        # 131072^2 float4 pixels = 256 GiB: more than the device holds.
        job = sv.submit(workloads.cornell(), width=131072, height=131072, spp=1, film=False)
        with pytest.raises(serve.JobError, match="more device memory"):
            job.wait()
        assert sv.stats().jobs_failed == 1


def test_cancel_queued_and_running(lib):
    with serve.Server(max_jobs=1, iteration_paths=1 << 15, tile=32, pass_spp=1) as sv:
        long_job = sv.submit(workloads.cornell(), width=256, height=256, spp=64)
        queued = sv.submit(workloads.cornell(), width=64, height=64, spp=4)
        queued.cancel()
        with pytest.raises(serve.JobError, match="cancelled"):
            queued.wait()
        long_job.cancel()
        with pytest.raises(serve.JobError, match="cancelled"):
            long_job.wait()
        st = sv.stats()
        assert st.jobs_cancelled == 2 and st.active_jobs == 0
        # The server keeps serving after cancellations.
        ok = sv.submit(workloads.cornell(), width=32, height=32, spp=2).wait()
        assert np.isfinite(ok).all()


def test_single_slot_serialises_jobs(lib):
    with serve.Server(max_jobs=1) as sv:
        a = sv.submit(workloads.cornell(), width=128, height=128, spp=8)
        b = sv.submit(workloads.cornell(), width=128, height=128, spp=8, seed=5)
        a.wait()
        b.wait()
        # b waits for a's slot: admitted only after a ended (b was submitted
        # a few milliseconds after a).
        assert b.last.queued_ms >= a.last.latency_ms - 50.0
        assert b.last.latency_ms > a.last.latency_ms
        assert sv.stats().scenes_resident == 1


def test_servers_and_sessions_share_a_device(lib, asset_dir):
    """Two servers on one device (what MultiServer does across devices, here
    on the one GPU a test gets) and a session rendering from this thread at
    the same time: each film is the one its job gets alone. The launch
    blocks all three use live in the device's constant memory; the
    per-device launch lock orders their batches and chunks."""
    import threading
    jobs = mix(asset_dir)
    cfg = dict(tile=32, pass_spp=4, iteration_paths=1 << 16, engine=0)
    alone = []
    for s, o in jobs:
        with serve.Server(**cfg) as sv:
            alone.append(sv.submit(s, base_dir=asset_dir, **o).wait())
    sref = session_film(workloads.cornell(), ".", engine=0, width=160, height=120, spp=16)
    ms = serve.MultiServer(devices=[0, 0], **cfg)
    try:
        handles = [ms.submit(s, base_dir=asset_dir, **o) for s, o in jobs]
        assert sorted(set(h.placement for h in handles)) == [0, 1]
        out = {}

        def session_renders():
            out["films"] = [session_film(workloads.cornell(), ".", engine=0, width=160,
                                         height=120, spp=16) for _ in range(3)]
        t = threading.Thread(target=session_renders)
        t.start()
        films = [h.wait() for h in handles]
        t.join()
    finally:
        ms.close()
    for f, a in zip(films, alone):
        assert np.array_equal(f, a)
    for f in out["films"]:
        assert np.array_equal(f, sref)


def test_multi_server_on_every_device(lib):
    """MultiServer over all visible devices (one here): jobs complete and
    equal the plain server's films."""
    s = workloads.cornell()
    with serve.Server() as sv:
        ref = sv.submit(s, width=64, height=64, spp=4).wait()
    with serve.MultiServer() as ms:
        assert len(ms.servers) == lib.sundog_device_count() >= 1
        film = ms.submit(s, width=64, height=64, spp=4).wait()
    assert np.array_equal(film, ref)
