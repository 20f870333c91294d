"""The compressed 8-wide BVH build (lib/libsundog_cw8.so: child boxes as 8-bit
offsets on a per-node grid, rounded outward so no hit is lost; final hit tests
in FP32) against the CPU oracle.

The variant library has the same ABI; the whole-image parity tests of
tests/test_gpu_render.py run against it in a fresh process (the library is
chosen at load time through SUNDOG_B200_LIB), with the same bounds. The
default build's binary BVH is the one the rest of the suite checks."""

import os
import subprocess
import sys

import pytest

from sundog_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_wide_bvh_image_parity():
    if not os.path.isfile(build.LIB_CW8):
        build.build(defines=("SDB_WIDE_BVH=1",), out=build.LIB_CW8)
    env = dict(os.environ, SUNDOG_B200_LIB=build.LIB_CW8)
    r = subprocess.run([sys.executable, "-m", "pytest", os.path.join(ROOT, "tests",
                                                                     "test_gpu_render.py"),
                        "-q", "-p", "no:cacheprovider", "-k", "parity or wavefront_matches"],
                       cwd=ROOT, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=900)
    print(r.stdout[-3000:])
    assert r.returncode == 0, r.stdout[-3000:]
    assert " passed" in r.stdout and "failed" not in r.stdout
