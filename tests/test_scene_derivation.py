"""The product's scene derivation against sundog's own scene code (CPU).

sundog derives the renderable scene from the C-ABI calls in
src/capi_scene.cpp and src/scene_build.cpp: defaults, transform composition
(scene_build.cpp:48-70), NEE registration of emissive quadrics and meshes
(scene_build.cpp:72-153) and the two point lights of each flame
(scene_build.cpp:155-181). The oracle compiles those two files unchanged into
oracle/_ref/libsdref_scene.so; the image parity tests take the oracle's scene
from there. This file checks that the product's own derivation
(sundog_scene_debug_json) writes the same oracle description, float for
float (%.9g of the FP32 values), for the benchmark workloads, the feature
scene and the call streams sundog's unchanged scenelib sends for its golden
scenes."""

import ctypes
import json
import os

import pytest

from oracle import oracle
from sundog_b200 import abi, workloads
from sundog_b200 import scene as sc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def product_text(lib, h, base_dir):
    text, _ = oracle.scene_text(sc.debug_json(h, lib), base_dir)
    return text


def reference_text_of(handle):
    rl = oracle.ref_scene_lib()
    need = ctypes.c_size_t(0)
    assert rl.sdo_ref_scene_text(handle, None, 0, ctypes.byref(need)) == 0
    buf = ctypes.create_string_buffer(need.value)
    rl.sdo_ref_scene_text(handle, buf, need.value, ctypes.byref(need))
    return buf.value.decode()


def assert_same(name, ref, ours):
    a, b = ref.strip().split("\n"), ours.strip().split("\n")
    assert len(a) == len(b), "%s: %d reference lines, %d here" % (name, len(a), len(b))
    diff = [(i, x, y) for i, (x, y) in enumerate(zip(a, b)) if x != y]
    assert not diff, "%s: %d lines differ, first %r" % (name, len(diff), diff[0])


@pytest.mark.parametrize("which", ["cornell", "instancing", "volumes", "features", "textured"])
def test_workload_derivation_matches_reference(lib, asset_dir, which):
    s = {"cornell": lambda: workloads.cornell(),
         "instancing": lambda: workloads.instancing(asset_dir),
         "volumes": lambda: workloads.volumes(asset_dir),
         "features": lambda: workloads.features(),
         "textured": lambda: workloads.textured(asset_dir)}[which]()
    ref, _ = oracle.reference_scene_text(s, asset_dir)
    h = s.build(asset_dir, lib)
    try:
        ours = product_text(lib, h, asset_dir)
    finally:
        lib.sundog_scene_destroy(h)
    assert_same(which, ref, ours)


def _decode(a, handle):
    if isinstance(a, dict):
        if "h" in a:
            return handle
        if "s" in a:
            return b"."
        if "d" in a:
            return (ctypes.c_double * len(a["d"]))(*a["d"])
        if "xf" in a:
            return (abi.XformStep * len(a["xf"]))(*[abi.XformStep(**f) for f in a["xf"]])
        if "pb" in a:
            f = dict(a["pb"])
            for k in ("velocity", "angular_velocity"):
                f[k] = (ctypes.c_double * 3)(*f[k])
            return ctypes.byref(abi.PhysicsBody(**f))
        raise ValueError(a)
    return a


def _replay(l, calls):
    h = None
    for name, args, ret in calls:
        r = getattr(l, name)(*[_decode(a, h) for a in args])
        if name == "sundog_scene_create":
            h = r
        else:
            assert r == ret, (name, r, ret)
    return h


@pytest.mark.parametrize("scene", ["smoke", "01-marble-run", "02-cornell-lume"])
def test_golden_call_streams_derive_as_reference(lib, scene):
    with open(os.path.join(GOLDEN, "abi_%s.json" % scene)) as f:
        calls = json.load(f)["calls"]
    rl = oracle.ref_scene_lib()
    hr = _replay(rl, calls)
    try:
        ref = reference_text_of(hr)
    finally:
        rl.sundog_scene_destroy(hr)
    hp = _replay(lib, calls)
    try:
        ours = product_text(lib, hp, ".")
    finally:
        lib.sundog_scene_destroy(hp)
    assert_same(scene, ref, ours)


def test_reference_scene_errors_match(lib):
    """An out-of-order call is rejected by both with the same message."""
    rl = oracle.ref_scene_lib()
    for l in (rl, lib):
        h = l.sundog_scene_create(b".")
        try:
            d3 = (ctypes.c_double * 3)(1, 1, 1)
            assert l.sundog_add_point_light(h, d3, d3, float("nan")) == 0
            rc = l.sundog_add_material_lambert(h, d3, -1)
            assert rc == -1
        finally:
            l.sundog_scene_destroy(h)
    assert abi.last_error(rl) == abi.last_error(lib)
