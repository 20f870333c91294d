"""Sampling tables built on the device (cdf_build.cu) against the FP64 host
oracle (oracle/tables.py, pinned to the CPU oracle's build of the reference's
loops by tests/test_oracle_tables.py).

Per table and quantity, printed: the share of entries bit-identical to the
reference-order table (sequential FP64 prefix sums; the device scans in
parallel, so a prefix can differ in its last FP64 bits and, next to a float
rounding boundary, in the stored float), and the maximum relative error
against the unrounded FP64 values (prefix / total). Bounds: >= 99.9% of
entries identical, relative error <= 1e-6 (a few FP32 ulps) for every entry.
The CDF index chosen for a given uniform is checked bit-exactly elsewhere
(tests/test_gpu_functions.py)."""

import ctypes
import os

import numpy as np
import pytest

from oracle import oracle, tables
from sundog_b200 import abi, workloads
from sundog_b200 import scene as sc

pytestmark = pytest.mark.gpu

REL = 1e-6
IDENTICAL = 0.999


def device_table(lib, ses, which):
    n = ctypes.c_size_t(0)
    abi.check(lib.sundog_session_table(ses.handle, which, None, 0, ctypes.byref(n)), "table", lib)
    out = np.zeros(n.value, np.float32)
    abi.check(lib.sundog_session_table(ses.handle, which, out.ctypes.data, n.value,
                                       ctypes.byref(n)), "table", lib)
    return out


def check_table(name, got, ref32, ref64):
    got = np.asarray(got, np.float32).ravel()
    ref32 = np.asarray(ref32, np.float32).ravel()
    ref64 = np.asarray(ref64, np.float64).ravel()
    assert got.shape == ref32.shape
    same = np.mean(got == ref32)
    nz = ref64 > 0
    rel = np.abs(got[nz].astype(np.float64) - ref64[nz]) / ref64[nz]
    print("%-28s n=%7d  identical to reference order %.6f  max rel err vs FP64 %.2e"
          % (name, got.size, same, rel.max() if rel.size else 0.0))
    assert same >= IDENTICAL, name
    assert rel.max() <= REL, name
    assert got[0] == 0.0 and got[-1] == 1.0


def test_env_cdf_tables(lib, asset_dir):
    s = workloads.instancing(asset_dir, width=32, height=18, spp=1)
    with sc.Session(s, base_dir=asset_dir) as ses:
        marg = device_table(lib, ses, 0)
        cond = device_table(lib, ses, 1)
    m, c, m64, c64 = tables.env_tables(tables.read_rgbe(os.path.join(asset_dir,
                                                                     "sky_1024x512.hdr")))
    check_table("env marginal CDF (513)", marg, m, m64)
    check_table("env conditional CDFs", cond, c, c64)
    # every row of the conditional table ends at 1
    assert np.all(cond.reshape(512, 1025)[:, -1] == 1.0)


def test_mesh_light_cdf_table(lib, asset_dir):
    s = workloads.volumes(asset_dir, width=32, height=18, spp=1)
    text, _ = oracle.reference_scene_text(s, asset_dir)
    obj = [l.split() for l in text.split("\n") if l.startswith("object 5")][0]
    light, xf = int(obj[6]), [float(x) for x in obj[7:19]]
    with sc.Session(s, base_dir=asset_dir) as ses:
        got = device_table(lib, ses, 2 + light)
        other = device_table(lib, ses, 2 + light + 1)
    pos, tris = tables.read_obj_triangles(os.path.join(asset_dir, "canopy_2048.obj"))
    cdf, cdf64, _ = tables.mesh_light_cdf(pos, tris, xf)
    check_table("mesh light area CDF (2049)", got, cdf, cdf64)
    assert other.size == 0  # the flame's point lights have no table


def test_black_env_rows_get_uniform_ramps(lib, tmp_path):
    """An env map with black rows (and one all-black map): uniform ramps,
    as the reference stores them."""
    rgb = np.zeros((16, 32, 3), np.float32)
    rgb[4:9] = np.linspace(0.1, 3.0, 32, dtype=np.float32)[None, :, None]
    workloads.write_hdr(str(tmp_path / "bands.hdr"), rgb)
    s = sc.Scene()
    s.render(width=8, height=8, spp=1)
    s.camera(lookfrom=[0, 0, 4], lookat=[0, 0, 0])
    s.background_envmap("bands.hdr")
    s.lambert("grey", color=[0.5, 0.5, 0.5])
    s.add("sphere", "grey")
    with sc.Session(s, base_dir=str(tmp_path)) as ses:
        marg = device_table(lib, ses, 0)
        cond = device_table(lib, ses, 1)
    m, c, m64, c64 = tables.env_tables(tables.read_rgbe(str(tmp_path / "bands.hdr")))
    check_table("banded env marginal", marg, m, m64)
    check_table("banded env conditional", cond, c, c64)
