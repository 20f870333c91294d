"""The 8-wide BVH builder on the host: every primitive is referenced once,
every quantised child box (8-bit grid, outward rounding) contains the exact
bounds of its subtree, leaves hold 1..3 primitives."""

import ctypes

import numpy as np
import pytest

from sundog_b200 import abi, workloads


def validate(lib, boxes, leaf_max=3):
    lib.sundog_bvh_validate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p]
    b = np.ascontiguousarray(boxes, np.float32)
    out = np.zeros(6, np.uint64)
    assert lib.sundog_bvh_validate(b.ctypes.data, len(b), leaf_max, out.ctypes.data) == 0
    return dict(zip(["nodes", "depth", "leaves", "inner", "slots", "fails"], out.tolist()))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 8, 9, 64, 1000, 20000])
def test_random_boxes(lib, n):
    rng = np.random.default_rng(n)
    c = rng.uniform(-50, 50, (n, 3))
    e = rng.exponential(0.5, (n, 3))
    r = validate(lib, np.concatenate([c - e, c + e], 1))
    assert r["fails"] == 0, r
    assert r["leaves"] >= (n + 2) // 3


def test_degenerate_and_flat_boxes(lib):
    n = 500
    rng = np.random.default_rng(3)
    c = rng.uniform(-1, 1, (n, 3))
    c[:, 1] = 0.0                      # all in one plane, zero y extent
    b = np.concatenate([c, c], 1)      # points
    assert validate(lib, b)["fails"] == 0
    same = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (50, 1))  # identical boxes
    assert validate(lib, same)["fails"] == 0


def test_icosphere_triangles(lib):
    v, f = workloads.icosphere(4)
    tri = v[f]
    boxes = np.concatenate([tri.min(1), tri.max(1)], 1)
    r = validate(lib, boxes)
    assert r["fails"] == 0 and len(f) == 5120
    assert r["depth"] <= 8
