"""Device memory of one-shot renders.

sundog's own render is self-contained: every device buffer it allocates is
freed before sundog_render returns (src/capi_render.cpp:65, 303-304). Here
the same holds by default; with the device-memory cache on
(sundog_set_device_memory_cache(1)) the per-sample buffer and the path pool
of a finished render stay allocated for the next call until
sundog_release_device_memory() frees them."""

import ctypes

import numpy as np
import pytest

from sundog_b200 import abi, workloads

pytestmark = pytest.mark.gpu

SLACK = 8 << 20  # allocator granularity and the driver's own bookkeeping


def free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def one_shot(lib, scene, base_dir="."):
    h = scene.build(base_dir, lib)
    try:
        film = np.zeros((scene._render["height"], scene._render["width"], 4), np.float32)
        o = abi.options(quiet=True)
        ext = abi.RenderExt(film.ctypes.data, None, None, 0, 1, 0, 0, 0, 0)
        res = abi.RenderResult()
        abi.check(lib.sundog_render_ex(h, ctypes.byref(o), ctypes.byref(ext), ctypes.byref(res)),
                  "render", lib)
    finally:
        lib.sundog_scene_destroy(h)
    return film


def test_one_shot_render_returns_device_memory(lib, asset_dir):
    s = workloads.instancing(asset_dir, width=640, height=360, spp=8)
    abi.check(lib.sundog_set_device_memory_cache(0), "cache", lib)
    one_shot(lib, s, asset_dir)  # first call: module load, context
    before = free_bytes()
    one_shot(lib, s, asset_dir)
    after = free_bytes()
    print("free before %.1f MiB, after %.1f MiB" % (before / 2**20, after / 2**20))
    assert abs(after - before) <= SLACK


def test_memory_cache_keeps_then_releases(lib, asset_dir):
    s = workloads.instancing(asset_dir, width=640, height=360, spp=8)
    abi.check(lib.sundog_set_device_memory_cache(0), "cache", lib)
    base = free_bytes()
    try:
        abi.check(lib.sundog_set_device_memory_cache(1), "cache", lib)
        a = one_shot(lib, s, asset_dir)
        held = base - free_bytes()
        b = one_shot(lib, s, asset_dir)  # reuses the kept buffers
        assert a.tobytes() == b.tobytes()
        assert base - free_bytes() <= held + SLACK
        print("held between calls: %.1f MiB" % (held / 2**20))
        assert held > 64 << 20
        abi.check(lib.sundog_release_device_memory(), "release", lib)
        assert abs(free_bytes() - base) <= SLACK
    finally:
        abi.check(lib.sundog_set_device_memory_cache(0), "cache", lib)
