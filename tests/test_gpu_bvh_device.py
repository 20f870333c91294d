"""BVHs built on the device (bvh_device.cu, the default) against the host
binned-SAH builder (sundog_set_bvh_builder(0)).

Both builders apply the same split rules (binned SAH over 32 bins per axis,
exact sweeps for ranges of up to 32 primitives, the same leaf rule); their
trees differ only where partitions break ties differently, so a ray visits
different nodes but finds the same closest accepted hit, up to primitives hit
at exactly the same distance. Bounds: >= 99.9% of pixels within 1e-3
relative, image relMSE <= 1e-6, ray counts within 0.05%; traversal work per
ray (counting build) within 10% of the host tree's."""

import ctypes

import numpy as np
import pytest

from sundog_b200 import abi, workloads
from sundog_b200 import scene as sc

pytestmark = pytest.mark.gpu


def render(lib, s, base_dir, device):
    abi.check(lib.sundog_set_bvh_builder(1 if device else 0), "builder", lib)
    try:
        with sc.Session(s, base_dir=base_dir) as ses:
            r = ses.render()
            film = ses.read()
            st = ses.stats
            cnt = abi.TraceCounts()
            abi.check(lib.sundog_session_trace_counts(ses.handle, ctypes.byref(cnt)), "counts", lib)
        return film, r, st, cnt
    finally:
        abi.check(lib.sundog_set_bvh_builder(1), "builder", lib)


@pytest.mark.parametrize("name", ["cornell", "instancing", "volumes", "features", "textured"])
def test_device_bvh_matches_host_bvh(lib, asset_dir, name):
    s = {"cornell": lambda: workloads.cornell(width=96, height=96, spp=8),
         "instancing": lambda: workloads.instancing(asset_dir, width=160, height=90, spp=4),
         "volumes": lambda: workloads.volumes(asset_dir, width=160, height=90, spp=4),
         "features": lambda: workloads.features(),
         "textured": lambda: workloads.textured(asset_dir)}[name]()
    fd, rd, sd, cd = render(lib, s, asset_dir, True)
    fh, rh, sh, ch = render(lib, s, asset_dir, False)
    g, o = fd[..., :3].astype(np.float64), fh[..., :3].astype(np.float64)
    scale = np.maximum(np.maximum(np.abs(g), np.abs(o)), 1e-2)
    frac = np.all(np.abs(g - o) <= 1e-3 * scale, axis=-1).mean()
    relmse = np.mean((g - o) ** 2) / max(np.mean(o ** 2), 1e-12)
    bd = cd.box_tests / max(cd.rays, 1)
    bh = ch.box_tests / max(ch.rays, 1)
    print("%s: device nodes %d depth %d/%d, host nodes %d depth %d/%d; pixels matching %.5f, "
          "relMSE %.2e; rays %d vs %d; box tests per ray %.2f vs %.2f"
          % (name, sd.bvh_nodes, sd.tlas_depth, sd.blas_depth, sh.bvh_nodes, sh.tlas_depth,
             sh.blas_depth, frac, relmse, rd.rays_traced, rh.rays_traced, bd, bh))
    assert frac >= 0.999
    assert relmse <= 1e-6
    assert abs(rd.rays_traced - rh.rays_traced) <= 5e-4 * rh.rays_traced
    assert bd <= 1.1 * bh
