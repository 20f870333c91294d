"""Scene-construction semantics of the C ABI, without a GPU.

Restates the checks of sundog's tests/host/test_scene_build.cpp (cited per
test) against libsundog.so, reading the derived state back through
sundog_scene_debug_json: defaults, the smoke scene call for call, error
paths and their messages, flames, water, plastic, envmap, the light-order
contract and phase guard, mesh-light placeholders, mirroring, the material
cap and the camera frame.
"""

import ctypes
import math

import pytest

from sundog_b200 import abi
from sundog_b200.scene import debug_json

NAN = float("nan")


def D3(x, y, z):
    return abi.c_d3(x, y, z)


def D2(x, y):
    return (ctypes.c_double * 2)(x, y)


def steps(*st):
    arr = (abi.XformStep * max(len(st), 1))()
    for i, s in enumerate(st):
        arr[i] = abi.XformStep(*s)
    return arr, len(st)


@pytest.fixture
def L(lib):
    return lib


def mini(L):
    h = L.sundog_scene_create(b"scenes")
    assert h
    assert L.sundog_set_camera(h, D3(0, 1, 5), D3(0, 0, 0), None, NAN, NAN, NAN) == 0
    assert L.sundog_add_material_lambert(h, D3(0.5, 0.5, 0.5), -1) == 0
    return h


def add_sphere(L, h, mat):
    return L.sundog_add_object(h, 0, -1, mat, -2, -1, None, 0, -1, None)


def expect_fail(L, rc, setter=False):
    if setter:
        assert rc != 0
    else:
        assert rc == -1
    msg = abi.last_error(L)
    assert msg
    return msg


def near(a, b, eps):
    return abs(a - b) <= eps


def test_minimal_defaults(L):  # test_scene_build.cpp:59-81
    h = mini(L)
    assert add_sphere(L, h, 0) == 0
    assert L.sundog_scene_validate(h) == 0
    s = debug_json(h)
    assert s["render"]["width"] == 1280 and s["render"]["height"] == 720
    assert s["render"]["spp"] == 64 and s["render"]["max_depth"] == 16
    assert s["render"]["clamp"] == 50 and s["render"]["seed"] == 7
    assert s["render"]["transparent_shadows"] == 1
    assert len(s["objects"]) == 1 and not s["lights"]
    assert s["base_dir"] == "scenes"
    h2 = L.sundog_scene_create(None)
    assert L.sundog_scene_validate(h2) != 0
    assert "missing camera" in abi.last_error(L)
    assert debug_json(h2)["base_dir"] == "."
    L.sundog_scene_destroy(h2)
    h3 = mini(L)
    assert L.sundog_set_render(h3, -1, -1, -1, -1, NAN, -1, NAN, 0) == 0
    assert debug_json(h3)["render"]["transparent_shadows"] == 0
    L.sundog_scene_destroy(h3)
    L.sundog_scene_destroy(h)


def test_smoke_equivalent(L):  # test_scene_build.cpp:85-158 (scenes/smoke.py)
    h = L.sundog_scene_create(b"scenes")
    assert L.sundog_set_render(h, 256, 256, 16, 8, NAN, 7, NAN, -1) == 0
    assert L.sundog_set_camera(h, D3(0, 1.5, 5), D3(0, 0.7, 0), None, 35.0, NAN, NAN) == 0
    assert L.sundog_set_background_gradient(h, D3(1, 1, 1), D3(0.4, 0.6, 1.0)) == 0
    assert L.sundog_add_texture_checker(h, D3(0.85, 0.85, 0.85), D3(0.15, 0.15, 0.15),
                                        D2(8, 8)) == 0
    ball = L.sundog_add_material_lambert(h, D3(0.7, 0.3, 0.3), -1)
    ground = L.sundog_add_material_lambert(h, None, 0)
    assert (ball, ground) == (0, 1)
    a, n = steps((0, 4, 4, 4))
    assert L.sundog_add_object(h, 1, -1, ground, -2, -1, a, n, -1, None) == 0
    a, n = steps((0, 0.7, 0.7, 0.7), (1, 0, 0.7, 0))
    assert L.sundog_add_object(h, 0, -1, ball, -2, -1, a, n, -1, None) == 1
    assert L.sundog_add_point_light(h, D3(3, 4, 2), D3(40, 40, 40), 0.4) == 0
    assert L.sundog_scene_validate(h) == 0
    s = debug_json(h)
    r = s["render"]
    assert (r["width"], r["height"], r["spp"], r["max_depth"], r["seed"]) == (256, 256, 16, 8, 7)
    assert near(s["camera"]["lookfrom"][1], 1.5, 1e-6) and near(s["camera"]["vfov"], 35, 1e-6)
    assert s["background"]["kind"] == 1
    assert near(s["background"]["a"][0], 1.0, 1e-6) and near(s["background"]["b"][2], 1.0, 1e-6)
    assert len(s["objects"]) == 2 and len(s["lights"]) == 1 and len(s["materials"]) == 2
    assert s["textures"][0]["kind"] == 2 and near(s["textures"][0]["scale"][0], 8, 1e-6)
    assert s["materials"][1]["tex"] == 0 and near(s["materials"][0]["color"][0], 0.7, 1e-6)
    x0, x1 = s["objects"][0]["xform"], s["objects"][1]["xform"]
    assert s["objects"][0]["kind"] == 1 and s["objects"][1]["kind"] == 0
    assert near(x0[0], 4.0, 1e-5)                        # applyVector(1,0,0).x
    assert near(x1[7], 0.7, 1e-5)                        # applyPoint(0,0,0).y
    assert near(math.sqrt(x1[0] ** 2 + x1[4] ** 2 + x1[8] ** 2), 0.7, 1e-5)
    assert s["objects"][0]["light"] == -1 and s["objects"][1]["light"] == -1
    l0 = s["lights"][0]
    assert l0["kind"] == 3 and near(l0["radius"], 0.4, 1e-6) and near(l0["p"][0], 3, 1e-6)
    assert near(l0["L"][0], 40, 1e-5)
    assert s["objects"][0]["mat_front"] == s["objects"][0]["mat_back"] != 0xFFFF
    L.sundog_scene_destroy(h)


def test_error_paths(L):  # test_scene_build.cpp:247-356
    h = mini(L)
    assert "texture id out of range" in expect_fail(L, L.sundog_add_material_lambert(h, None, 7))
    expect_fail(L, L.sundog_add_material_emissive(h, D3(1, 1, 1), -1, -2.0, -1))
    assert "unknown shape" in expect_fail(L, L.sundog_add_object(h, 99, -1, 0, -2, -1, None, 0,
                                                                 -1, None))
    assert "mesh id out of range" in expect_fail(L, L.sundog_add_object(h, 5, 3, 0, -2, -1, None,
                                                                        0, -1, None))
    assert "material id out of range" in expect_fail(L, add_sphere(L, h, 42))
    assert "no material on either face" in expect_fail(
        L, L.sundog_add_object(h, 0, -1, -1, -1, -1, None, 0, -1, None))
    assert "cutout texture id out of range" in expect_fail(
        L, L.sundog_add_object(h, 0, -1, 0, -2, 5, None, 0, -1, None))
    a, n = steps((99, 1, 1, 1))
    assert "unknown transform step kind" in expect_fail(
        L, L.sundog_add_object(h, 0, -1, 0, -2, -1, a, n, -1, None))
    expect_fail(L, L.sundog_add_point_light(h, D3(0, 5, 0), D3(10, -1, 10), 0.0))
    expect_fail(L, L.sundog_add_distant_light(h, D3(0, -1, 0), D3(-0.1, 1, 1)))
    L.sundog_scene_destroy(h)

    h = L.sundog_scene_create(None)
    g = L.sundog_add_material_dielectric(h, NAN, D3(0.4, 0.05, 0.02), None, -1, NAN)
    p = L.sundog_add_material_dielectric(h, NAN, None, None, -1, NAN)
    fr = L.sundog_add_material_dielectric(h, NAN, None, None, -1, 0.35)
    assert (g, p, fr) == (0, 1, 2)
    m = debug_json(h)["materials"]
    assert near(m[0]["absorb"][0], 0.4, 1e-6) and m[1]["absorb"][0] == 0.0
    assert m[0]["roughness"] == 0.0 and near(m[2]["roughness"], 0.35, 1e-6)
    assert near(m[0]["ior"], 1.5, 1e-6)
    expect_fail(L, L.sundog_add_material_dielectric(h, NAN, D3(-0.1, 0, 0), None, -1, NAN))
    L.sundog_scene_destroy(h)

    h = mini(L)
    em = L.sundog_add_material_emissive(h, None, -1, 5.0, -1)
    se = L.sundog_add_material_emissive(h, D3(1, 1, 1), -1, 3.0, -1)
    tex = L.sundog_add_texture_image(h, b"textures/spot_texture.avif", -1)
    tem = L.sundog_add_material_emissive(h, None, tex, 2.0, -1)
    assert min(em, se, tex, tem) >= 0
    a, n = steps((0, 2, 1, 1))
    assert "uniform XZ scale" in expect_fail(L, L.sundog_add_object(h, 2, -1, em, -2, -1, a, n,
                                                                     -1, None))
    assert "uniform scale" in expect_fail(L, L.sundog_add_object(h, 0, -1, em, -2, -1, a, n, -1,
                                                                  None))
    assert L.sundog_add_object(h, 2, -1, em, -2, -1, a, n, 0, None) >= 0
    s = debug_json(h)
    assert not s["lights"] and s["objects"][-1]["light"] == -1 and s["objects"][-1]["nee"] == 0
    a, n = steps((0, 2, 2, 2), (1, 1, 5, 0))
    assert L.sundog_add_object(h, 0, -1, se, -2, -1, a, n, -1, None) >= 0
    s = debug_json(h)
    l0 = s["lights"][0]
    assert len(s["lights"]) == 1 and l0["kind"] == 2
    assert near(l0["radius"], 2.0, 1e-5) and near(l0["p"][1], 5.0, 1e-5)
    assert near(l0["L"][0], 3.0, 1e-5) and s["objects"][-1]["light"] == 0
    a, n = steps((0, 1, 1, 1))
    assert "textured emissive sphere" in expect_fail(
        L, L.sundog_add_object(h, 0, -1, tem, -2, -1, a, n, -1, None))
    assert L.sundog_add_object(h, 4, -1, -1, 0, -1, None, 0, -1, None) >= 0
    s = debug_json(h)
    assert s["objects"][-1]["mat_front"] == 0xFFFF and s["objects"][-1]["mat_back"] != 0xFFFF
    assert L.sundog_add_object(h, 1, -1, 0, -2, tex, None, 0, -1, None) >= 0
    s = debug_json(h)
    assert s["textures"][s["objects"][-1]["cutout"]]["kind"] == 1
    L.sundog_scene_destroy(h)


def test_flames(L):  # test_scene_build.cpp:457-500
    h = mini(L)
    a, n = steps((0, 8, 8, 8))
    assert L.sundog_add_object(h, 1, -1, 0, -2, -1, a, n, -1, None) >= 0
    assert L.sundog_add_flame(h, D3(1, 0.2, -1), 1.5, 0.4, 25, 5, 2.5, 7, 16) == 0
    s = debug_json(h)
    f = s["flames"][0]
    assert near(f["base"][0], 1, 1e-6) and near(f["height"], 1.5, 1e-6)
    assert near(f["radius"], 0.4, 1e-6) and near(f["intensity"], 25, 1e-5)
    assert near(f["sigma"], 5, 1e-6) and near(f["noise_scale"], 2.5, 1e-6) and f["seed"] == 7
    assert f["steps"] == 32
    lt = s["lights"]
    assert len(lt) == 2 and lt[0]["kind"] == 3 and lt[1]["kind"] == 3
    assert near(lt[0]["p"][1], 0.2 + 0.35 * 1.5, 1e-5) and near(lt[1]["p"][1], 0.2 + 0.70 * 1.5, 1e-5)
    assert near(lt[0]["radius"], 0.12, 1e-6) and lt[0]["L"][0] > lt[1]["L"][0]
    assert near(lt[0]["L"][0], 16 * 0.65, 1e-5) and near(lt[1]["L"][1], 0.62 * 16 * 0.35, 1e-5)
    assert lt[0]["flame"] == 0 and lt[1]["flame"] == 0
    assert L.sundog_add_flame(h, D3(-2, 0, 1), 1.0, 0.3, NAN, NAN, NAN, -1, NAN) == 1
    lt = debug_json(h)["lights"]
    assert len(lt) == 4 and lt[2]["flame"] == 1 and lt[3]["flame"] == 1
    assert L.sundog_set_flame_steps(h, 1, 64) == 0
    assert debug_json(h)["flames"][1]["steps"] == 64
    assert L.sundog_set_flame_steps(h, 5, 64) != 0
    assert L.sundog_set_flame_steps(h, 0, 0) != 0
    L.sundog_scene_destroy(h)
    h = mini(L)
    assert add_sphere(L, h, 0) >= 0
    assert L.sundog_add_flame(h, D3(0, 0, 0), 1, 0.5, NAN, NAN, NAN, -1, NAN) == 0
    f = debug_json(h)["flames"][0]
    assert near(f["intensity"], 20, 1e-5) and near(f["sigma"], 4, 1e-6)
    assert near(f["noise_scale"], 3, 1e-6) and f["seed"] == 0
    expect_fail(L, L.sundog_add_flame(h, D3(0, 0, 0), 0, 0.5, NAN, NAN, NAN, -1, NAN))
    L.sundog_scene_destroy(h)


def test_water_plastic_envmap(L):  # test_scene_build.cpp:502-573
    h = L.sundog_scene_create(None)
    assert L.sundog_set_camera(h, D3(0, 2, 8), D3(0, 0, 0), None, NAN, NAN, NAN) == 0
    lake = L.sundog_add_material_water(h, NAN, None, NAN, NAN, None)
    pool = L.sundog_add_material_water(h, 1.34, D3(0.6, 0.1, 0.05), 0.12, 3.5, None)
    assert (lake, pool) == (0, 1)
    m = debug_json(h)["materials"]
    assert m[0]["kind"] == 4 and near(m[0]["ior"], 1.33, 1e-6)
    assert near(m[0]["absorb"][0], 0.45, 1e-6) and m[0]["absorb"][0] > m[0]["absorb"][1] > m[0]["absorb"][2]
    assert near(m[0]["wave_amp"], 0.05, 1e-6) and near(m[0]["wave_freq"], 2.0, 1e-6)
    assert near(m[0]["color"][0], 1.0, 1e-6)
    assert near(m[1]["ior"], 1.34, 1e-6) and near(m[1]["absorb"][1], 0.1, 1e-6)
    assert near(m[1]["wave_amp"], 0.12, 1e-6) and near(m[1]["wave_freq"], 3.5, 1e-6)
    expect_fail(L, L.sundog_add_material_water(h, NAN, None, -0.1, NAN, None))
    expect_fail(L, L.sundog_add_material_water(h, NAN, D3(-0.1, 0, 0), NAN, NAN, None))
    toy = L.sundog_add_material_plastic(h, D3(0.85, 0.2, 0.15), -1, NAN)
    matte = L.sundog_add_material_plastic(h, None, -1, 0.6)
    m = debug_json(h)["materials"]
    assert m[toy]["kind"] == 5 and near(m[toy]["roughness"], 0.15, 1e-6)
    assert near(m[toy]["ior"], 1.5, 1e-6) and near(m[matte]["roughness"], 0.6, 1e-6)
    assert not debug_json(h)["lights"]
    L.sundog_scene_destroy(h)

    h = mini(L)
    assert L.sundog_set_background_envmap(h, b"../assets/sky.hdr", 90, 2.5, 0) == 0
    b = debug_json(h)["background"]
    assert b["kind"] == 2 and b["env_file"] == "../assets/sky.hdr"
    assert near(b["env_rotate_deg"], 90, 1e-6) and near(b["env_intensity"], 2.5, 1e-6)
    assert b["env_importance"] == 0
    L.sundog_scene_destroy(h)
    h = mini(L)
    assert L.sundog_set_background_envmap(h, b"sky.hdr", NAN, NAN, -1) == 0
    b = debug_json(h)["background"]
    assert b["env_rotate_deg"] == 0 and b["env_intensity"] == 1 and b["env_importance"] == 1
    expect_fail(L, L.sundog_set_background_envmap(h, None, NAN, NAN, -1), setter=True)
    expect_fail(L, L.sundog_set_background_envmap(h, b"sky.hdr", NAN, -1.0, -1), setter=True)
    L.sundog_scene_destroy(h)


def test_light_order_and_phases(L):  # test_scene_build.cpp:578-617
    h = mini(L)
    mesh = L.sundog_add_mesh(h, b"../assets/sparky.obj", -1, b"EmitYellow")
    em = L.sundog_add_material_emissive(h, D3(1, 1, 1), -1, 4.0, -1)
    a, n = steps((0, 1, 1, 1))
    assert mesh == 0
    assert L.sundog_add_object(h, 1, -1, em, -2, -1, a, n, -1, None) >= 0
    assert L.sundog_add_object(h, 5, mesh, em, -2, -1, a, n, -1, None) >= 0
    assert L.sundog_add_flame(h, D3(0, 0, 0), 1, 0.5, NAN, NAN, NAN, -1, NAN) == 0
    assert L.sundog_add_point_light(h, D3(0, 5, 0), D3(10, 10, 10), NAN) >= 0
    lt = debug_json(h)["lights"]
    assert [l["kind"] for l in lt] == [0, 5, 3, 3, 3]
    assert near(lt[4]["p"][1], 5.0, 1e-6)
    assert [l["flame"] for l in lt] == [-1, -1, 0, 0, -1]
    assert "must come before" in expect_fail(L, L.sundog_add_object(h, 0, -1, 0, -2, -1, None,
                                                                     0, -1, None))
    expect_fail(L, L.sundog_add_flame(h, D3(0, 0, 0), 1, 0.5, NAN, NAN, NAN, -1, NAN))
    expect_fail(L, L.sundog_set_render(h, 64, 64, -1, -1, NAN, -1, NAN, -1), setter=True)
    expect_fail(L, L.sundog_add_material_lambert(h, None, -1))
    L.sundog_scene_destroy(h)


def test_mesh_light_placeholders(L):  # test_scene_build.cpp:623-693
    h = mini(L)
    mesh = L.sundog_add_mesh(h, b"../assets/sparky.obj", -1, b"EmitYellow")
    tex = L.sundog_add_texture_image(h, b"textures/spot_texture.avif", -1)
    em = L.sundog_add_material_emissive(h, D3(1.0, 0.85, 0.2), -1, 6.0, -1)
    tem = L.sundog_add_material_emissive(h, None, tex, 3.0, -1)
    a, n = steps((0, 2, 1, 3), (1, 0, 1, 0))
    assert L.sundog_add_object(h, 5, mesh, em, -2, -1, a, n, -1, None) >= 0
    s = debug_json(h)
    assert len(s["lights"]) == 1 and s["lights"][0]["kind"] == 5 and s["objects"][-1]["light"] == 0
    assert near(s["lights"][0]["L"][0], 6.0, 1e-5)
    assert s["lights"][0]["tex"] == -1 and s["lights"][0]["flame"] == -1
    assert L.sundog_add_object(h, 5, mesh, tem, -2, -1, a, n, -1, None) >= 0
    s = debug_json(h)
    assert s["lights"][1]["kind"] == 5 and s["lights"][1]["tex"] == tex
    assert near(s["lights"][1]["L"][0], 3.0, 1e-5)
    assert L.sundog_add_object(h, 5, mesh, em, -2, -1, a, n, 0, None) >= 0
    assert debug_json(h)["objects"][-1]["light"] == -1
    expect_fail(L, L.sundog_add_object(h, 5, mesh, em, -2, tex, a, n, -1, None))
    expect_fail(L, L.sundog_add_object(h, 1, -1, em, -2, tex, a, n, -1, None))
    assert len(debug_json(h)["lights"]) == 2
    assert L.sundog_add_object(h, 5, mesh, em, -2, tex, a, n, 0, None) >= 0
    L.sundog_scene_destroy(h)

    h = mini(L)
    assert L.sundog_set_physics(h, None, NAN, NAN, NAN, NAN, -1, -1, NAN, NAN) == 0
    mesh = L.sundog_add_mesh(h, b"../assets/spot.obj", -1, None)
    em = L.sundog_add_material_emissive(h, None, -1, 5.0, -1)
    dyn = abi.PhysicsBody(1, NAN, 0, 0, abi.c_d3(0, 0, 0), abi.c_d3(0, 0, 0), NAN, NAN, NAN)
    expect_fail(L, L.sundog_add_object(h, 5, mesh, em, -2, -1, None, 0, -1, ctypes.byref(dyn)))
    assert not debug_json(h)["lights"]
    L.sundog_scene_destroy(h)


def test_mirror_keeps_light_normal(L):  # test_scene_build.cpp:696-706
    h = mini(L)
    em = L.sundog_add_material_emissive(h, D3(1, 1, 1), -1, 2.0, -1)
    a, n = steps((0, -1, 1, 1))
    assert L.sundog_add_object(h, 1, -1, em, -2, -1, a, n, -1, None) >= 0
    l = debug_json(h)["lights"][-1]
    assert near(l["n"][1], 1.0, 1e-5) and near(l["area"], 4.0, 1e-5)
    L.sundog_scene_destroy(h)


def test_material_cap(L):  # test_scene_build.cpp:708-715
    h = L.sundog_scene_create(None)
    for i in range(0xFFFF):
        assert L.sundog_add_material_lambert(h, None, -1) == i
    assert "too many materials" in expect_fail(L, L.sundog_add_material_lambert(h, None, -1))
    L.sundog_scene_destroy(h)


def test_camera_frame(L):  # test_scene_build.cpp:717-734
    h = L.sundog_scene_create(None)
    assert L.sundog_set_render(h, 100, 100, -1, -1, NAN, -1, NAN, -1) == 0
    assert L.sundog_set_camera(h, D3(0, 0, 5), D3(0, 0, 0), D3(0, 1, 0), 90.0, NAN, NAN) == 0
    c = debug_json(h)["camera"]["frame"]
    assert near(c["w"][2], 1, 1e-5) and near(c["u"][0], 1, 1e-5) and near(c["v"][1], 1, 1e-5)
    assert near(c["origin"][2], 5, 1e-6)
    assert near(c["horizontal"][0], 10, 1e-4) and near(c["vertical"][1], 10, 1e-4)
    assert near(c["lower_left"][0], -5, 1e-4) and near(c["lower_left"][1], -5, 1e-4)
    assert near(c["lower_left"][2], 0, 1e-4) and c["lens_radius"] == 0
    L.sundog_scene_destroy(h)


def test_physics_block(L):  # test_scene_build.cpp:358-455 (registration only)
    h = mini(L)
    body = abi.PhysicsBody(0, NAN, 0, 0, abi.c_d3(0, 0, 0), abi.c_d3(0, 0, 0), NAN, NAN, NAN)
    assert "no top-level physics block" in expect_fail(
        L, L.sundog_add_object(h, 1, -1, 0, -2, -1, None, 0, -1, ctypes.byref(body)))
    L.sundog_scene_destroy(h)
    h = mini(L)
    assert L.sundog_set_physics(h, D3(0, -9.8, 0), 1 / 240.0, 8.0, 0.5, 0.2, 12, 3, NAN, 0.5) == 0
    p = debug_json(h)["physics"]
    assert p["enabled"] == 1 and near(p["gravity"][1], -9.8, 1e-6) and p["pos_iters"] == 12
    assert near(p["stop_time"], 0.5, 1e-6)
    dyn = abi.PhysicsBody(1, 300.0, 0, 0, abi.c_d3(0, 0, 0), abi.c_d3(0, 0, 0), NAN, NAN, NAN)
    assert "static-only" in expect_fail(
        L, L.sundog_add_object(h, 1, -1, 0, -2, -1, None, 0, -1, ctypes.byref(dyn)))
    assert "collider" in expect_fail(
        L, L.sundog_add_object(h, 3, -1, 0, -2, -1, None, 0, -1, ctypes.byref(dyn)))
    assert L.sundog_add_object(h, 0, -1, 0, -2, -1, None, 0, -1, ctypes.byref(dyn)) >= 0
    o = debug_json(h)["objects"][-1]
    assert o["physics"] == 1 and o["dynamic"] == 1 and near(o["density"], 300, 1e-4)
    expect_fail(L, L.sundog_set_physics(h, None, 0.0, NAN, NAN, NAN, -1, -1, NAN, NAN), setter=True)
    L.sundog_scene_destroy(h)


def test_render_argument_errors(L):
    h = mini(L)
    assert L.sundog_render(h, None) != 0
    assert "options" in abi.last_error(L) or "out_path" in abi.last_error(L)
    o = abi.options(out=None)
    assert L.sundog_render(h, ctypes.byref(o)) != 0
    assert "out_path is required" in abi.last_error(L)
    L.sundog_scene_destroy(h)
    h2 = L.sundog_scene_create(None)
    o = abi.options(out="/tmp/x.pfm")
    assert L.sundog_render(h2, ctypes.byref(o)) != 0
    assert "missing camera" in abi.last_error(L)
    L.sundog_scene_destroy(h2)
