"""Python front end of the render server (sundog_server_* in
include/sundog_api.h): submit scenes as jobs, wait for their films.

    with Server(max_jobs=16) as sv:
        job = sv.submit(scene, width=512, height=512, spp=64)
        film = job.wait()          # HxWx4 float32, bit-identical to a plain render

Several GPUs: MultiServer runs one server per device and places each job on
the device with the least queued camera paths (jobs are independent, so a
job's film is the one it would get alone on any device).

    with MultiServer() as ms:      # every visible device
        jobs = [ms.submit(s, width=1024, height=1024, spp=64) for s in scenes]
        films = [j.wait() for j in jobs]
"""

import ctypes

import numpy as np

from . import abi


class JobError(RuntimeError):
    """A job ended FAILED or CANCELLED."""


class Job(object):
    def __init__(self, server, job_id, film):
        self.server = server
        self.id = job_id
        self.film = film

    def status(self):
        st = abi.JobStatus()
        abi.check(self.server.lib.sundog_server_status(self.server.handle, self.id,
                                                       ctypes.byref(st)), "job status",
                  self.server.lib)
        return st

    def wait(self, timeout_ms=-1.0):
        """Blocks until the job ends; returns its film (raises JobError if it
        failed or was cancelled)."""
        st = abi.JobStatus()
        abi.check(self.server.lib.sundog_server_wait(self.server.handle, self.id, timeout_ms,
                                                     ctypes.byref(st)), "job wait",
                  self.server.lib)
        self.last = st
        self.server._live.pop(self.id, None)
        if st.state != abi.JOB_DONE:
            state = "failed" if st.state == abi.JOB_FAILED else "cancelled"
            raise JobError("job %d %s: %s" % (self.id, state, st.error.decode(errors="replace")))
        return self.film

    def cancel(self):
        abi.check(self.server.lib.sundog_server_cancel(self.server.handle, self.id), "cancel",
                  self.server.lib)


class Server(object):
    def __init__(self, device=None, **cfg):
        """device: the CUDA device of the server (None: the library's current
        device); cfg: sundog_server_config fields."""
        self.lib = abi.load()
        c = abi.ServerConfig()
        self.lib.sundog_server_defaults(ctypes.byref(c))
        for k, v in cfg.items():
            if not hasattr(c, k):
                raise TypeError("unknown server option %r" % k)
            setattr(c, k, v)
        self.config = c
        self.device = device
        # Host films of jobs not yet seen to end: the server writes into them.
        self._live = {}
        if device is None:
            self.handle = self.lib.sundog_server_create(ctypes.byref(c))
        else:
            self.handle = self.lib.sundog_server_create_on_device(ctypes.byref(c), int(device))
        if not self.handle:
            raise abi.SundogError("server: " + abi.last_error(self.lib))

    def submit(self, scene, base_dir=".", film=True, **opts):
        """Queues scene (a scene.Scene) with sundog_render-style overrides
        (width, height, spp, seed, ...). Returns a Job."""
        h = scene.build(base_dir, self.lib)
        try:
            o = abi.options(**opts)
            w = opts.get("width", -1)
            w = w if w > 0 else int(scene._render.get("width", 1280))
            ht = opts.get("height", -1)
            ht = ht if ht > 0 else int(scene._render.get("height", 720))
            buf = np.zeros((ht, w, 4), np.float32) if film else None
            jid = self.lib.sundog_server_submit(self.handle, h, ctypes.byref(o),
                                                buf.ctypes.data if film else None)
            if jid < 0:
                raise abi.SundogError("submit: " + abi.last_error(self.lib))
        finally:
            self.lib.sundog_scene_destroy(h)
        self._live[jid] = buf
        return Job(self, jid, buf)

    def stats(self):
        st = abi.ServerStatistics()
        abi.check(self.lib.sundog_server_stats(self.handle, ctypes.byref(st)), "stats", self.lib)
        return st

    def close(self):
        if getattr(self, "handle", None):
            self.lib.sundog_server_destroy(self.handle)
            self.handle = None
            self._live = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()


def least_loaded(loads):
    """Index of the smallest queued load (the first on ties)."""
    best = 0
    for i, x in enumerate(loads):
        if x < loads[best]:
            best = i
    return best


class MultiServer(object):
    """One Server per device; each submitted job goes to the device with the
    least queued camera paths (width x height x spp of its jobs not yet
    finished). Jobs are independent renders, so placement changes only when a
    film is ready, not what it holds. `servers` takes ready-made server
    objects (submit / stats / close, jobs with status()) in place of devices."""

    def __init__(self, devices=None, servers=None, **cfg):
        if servers is not None:
            self.servers = list(servers)
        else:
            if devices is None:
                n = abi.load().sundog_device_count()
                if n < 1:
                    raise abi.SundogError("server: no CUDA device")
                devices = list(range(n))
            self.servers = [Server(device=d, **cfg) for d in devices]
        self._queued = [[] for _ in self.servers]  # per server: [paths, job]

    def load(self, k):
        """Camera paths of the jobs on server k that have not finished."""
        live = [(p, j) for p, j in self._queued[k] if j.status().state < abi.JOB_DONE]
        self._queued[k] = live
        return sum(p for p, _ in live)

    def submit(self, scene, base_dir=".", film=True, **opts):
        k = least_loaded([self.load(i) for i in range(len(self.servers))])

        def opt(name, default):
            v = opts.get(name, -1)
            return v if v and v > 0 else int(scene._render.get(name, default))
        job = self.servers[k].submit(scene, base_dir=base_dir, film=film, **opts)
        self._queued[k].append([opt("width", 1280) * opt("height", 720) * opt("spp", 64), job])
        job.placement = k
        return job

    def stats(self):
        return [s.stats() for s in self.servers]

    def close(self):
        for s in self.servers:
            s.close()
        self.servers = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
