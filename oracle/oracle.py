"""ORACLE — test infrastructure only (the checker, never the product).

Python front end of the CPU oracle (oracle/_build/libsdoracle.so, built by
oracle/Makefile). The oracle's scene comes from the reference itself:
reference_scene_text() replays a scene's calls into sundog's own
scene-construction code (src/capi_scene.cpp + src/scene_build.cpp, compiled
into oracle/_ref/libsdref_scene.so by `make ref`), which derives the camera
settings, transforms, NEE light registration and flame lights, and writes the
result as the oracle's text description. The oracle loads that and renders
pixel rectangles on the host cores. scene_text() turns a library's
parse-time state (sundog_scene_debug_json) into the same description; the
tests use it only to compare the product's derivation with the reference's.
The module also exposes the oracle's function harness (sdo_fn) for
per-function parity checks.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsdoracle.so")
REF_FNVEC = os.path.join(HERE, "_ref", "fnvec_ref")
REF_SCENE_LIB = os.path.join(HERE, "_ref", "libsdref_scene.so")

_lib = None
_ref_scene = None


def build(force=False):
    """Compile the oracle with its Makefile, and the reference-built parts
    (function harness, scene library) when the reference sources are
    mounted."""
    import subprocess
    from oracle.refpath import reference_root
    targets = ["all"]
    ref = reference_root()
    if ref is not None:
        targets += ["ref", "REF=" + ref]
    if force:
        subprocess.run(["make", "-C", HERE, "clean"], check=True, stdout=subprocess.DEVNULL)
    subprocess.run(["make", "-C", HERE] + targets, check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


def ref_scene_lib():
    """sundog's own scene-construction library (oracle/_ref/libsdref_scene.so)
    with the scene ABI's prototypes declared. Raises when it was never built:
    it is built from the reference sources, which must be mounted once (the
    built library then travels with the repository)."""
    global _ref_scene
    if _ref_scene is None:
        if not os.path.isfile(REF_SCENE_LIB):
            build()
        if not os.path.isfile(REF_SCENE_LIB):
            raise RuntimeError("oracle: %s is not built (it compiles sundog's own "
                               "src/capi_scene.cpp and src/scene_build.cpp; mount the reference "
                               "and run oracle.build())" % REF_SCENE_LIB)
        from sundog_b200 import abi
        lib = ctypes.CDLL(REF_SCENE_LIB, mode=ctypes.RTLD_LOCAL)
        abi.declare_scene_abi(lib)
        lib.sdo_ref_scene_text.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t)]
        lib.sdo_ref_scene_forget.argtypes = [ctypes.c_void_p]
        lib.sdo_ref_scene_forget.restype = None
        _ref_scene = lib
    return _ref_scene


def apply_overrides(text, width=None, height=None, spp=None, seed=None, clamp=None,
                    transparent_shadows=None):
    """Applies sundog_render_options' overrides (src/capi_render.cpp:74-83:
    spp / width / height when > 0, seed when >= 0, clamp when set and >= 0,
    transparent shadows when >= 0) to the render line of an oracle
    description. Returns (text, render dict)."""
    lines = text.split("\n")
    f = lines[0].split()
    assert f[0] == "render", "oracle description must start with its render line"
    r = {"width": int(f[1]), "height": int(f[2]), "spp": int(f[3]), "max_depth": int(f[4]),
         "clamp": float(f[5]), "seed": int(f[6]), "transparent_shadows": int(f[7])}
    if width:
        r["width"] = width
    if height:
        r["height"] = height
    if spp:
        r["spp"] = spp
    if seed is not None and seed >= 0:
        r["seed"] = seed
    if clamp is not None and clamp >= 0:
        r["clamp"] = clamp
    if transparent_shadows is not None and transparent_shadows >= 0:
        r["transparent_shadows"] = transparent_shadows
    lines[0] = "render %d %d %d %d %s %d %d" % (r["width"], r["height"], r["spp"],
                                                 r["max_depth"], _f(r["clamp"]), r["seed"],
                                                 r["transparent_shadows"])
    return "\n".join(lines), r


def reference_scene_text(scene, base_dir, **overrides):
    """The oracle description of `scene` (a sundog_b200.scene.Scene: the
    scenelib-style call list) as sundog's own scene code derives it: the
    calls are replayed, in scenelib's order, into oracle/_ref/libsdref_scene.so
    and the derived sd::Scene is written out. Returns (text, render dict)
    with the render-option overrides applied."""
    lib = ref_scene_lib()
    h = scene.build(base_dir, lib)
    try:
        need = ctypes.c_size_t(0)
        if lib.sdo_ref_scene_text(h, None, 0, ctypes.byref(need)) != 0:
            raise RuntimeError("oracle: reference scene text failed")
        buf = ctypes.create_string_buffer(need.value)
        lib.sdo_ref_scene_text(h, buf, need.value, ctypes.byref(need))
        text = buf.value.decode()
    finally:
        lib.sdo_ref_scene_forget(h)
        lib.sundog_scene_destroy(h)
    return apply_overrides(text, **overrides)


def load():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.sdo_scene_load.restype = ctypes.c_void_p
        lib.sdo_scene_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        lib.sdo_scene_free.argtypes = [ctypes.c_void_p]
        lib.sdo_render.restype = ctypes.c_ulonglong
        lib.sdo_render.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [ctypes.c_void_p] * 3
        lib.sdo_scene_table.restype = ctypes.c_long
        lib.sdo_scene_table.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_long]
        lib.sdo_fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.sdo_quadric_fp64.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        _lib = lib
    return _lib


def fn(which, payload, n, out_dtype):
    """Run the oracle's restated function `which` over n packed items."""
    out = np.zeros(n, out_dtype)
    buf = ctypes.create_string_buffer(bytes(payload), len(payload))
    if load().sdo_fn(which, buf, n, out.ctypes.data) != 0:
        raise RuntimeError("oracle: unknown function %d" % which)
    return out


def quadric_fp64(kind, o, d, tmin=0.0, tmax=1e16):
    out = np.zeros(3, np.float64)
    oo = np.asarray(o, np.float64)
    dd = np.asarray(d, np.float64)
    load().sdo_quadric_fp64(kind, oo.ctypes.data, dd.ctypes.data, tmin, tmax, out.ctypes.data)
    return int(out[0]), out[1], out[2]


def _f(v):
    return "%.9g" % float(np.float32(v))


def _v(v):
    return " ".join(_f(c) for c in v)


def scene_text(state, base_dir, width=None, height=None, spp=None, seed=None, clamp=None,
               transparent_shadows=None):
    """Oracle text description from the parse-time scene state, with the
    render overrides of sundog_render_options (src/capi_render.cpp:74-83)."""
    r = dict(state["render"])
    if width:
        r["width"] = width
    if height:
        r["height"] = height
    if spp:
        r["spp"] = spp
    if seed is not None and seed >= 0:
        r["seed"] = seed
    if clamp is not None and clamp >= 0:
        r["clamp"] = clamp
    if transparent_shadows is not None and transparent_shadows >= 0:
        r["transparent_shadows"] = transparent_shadows

    def path(p):
        return p if os.path.isabs(p) else os.path.join(base_dir, p)

    c = state["camera"]
    lines = ["render %d %d %d %d %s %d %d" % (r["width"], r["height"], r["spp"], r["max_depth"],
                                              _f(r["clamp"]), r["seed"], r["transparent_shadows"]),
             "camera %s %s %s %s %s %s" % (_v(c["lookfrom"]), _v(c["lookat"]), _v(c["up"]),
                                           _f(c["vfov"]), _f(c["aperture"]), _f(c["focus_dist"]))]
    bg = state["background"]
    lines.append("bg %d %s %s" % (bg["kind"], _v(bg["a"]), _v(bg["b"])))
    if bg["kind"] == 2:
        lines.append("env %s %s %s %d" % (path(bg["env_file"]), _f(bg["env_rotate_deg"]),
                                          _f(bg["env_intensity"]), bg["env_importance"]))
    for t in state["textures"]:
        lines.append("texture %d %s %s %s %s %s %d %s" % (
            t["kind"], _v(t["a"]), _v(t["b"]), _f(t["scale"][0]), _f(t["scale"][1]),
            _f(t["width"]), t["srgb"], path(t["file"]) if t["file"] else "-"))
    for m in state["materials"]:
        lines.append("material %d %d %s %s %s %s %d %s %s %s" % (
            m["kind"], m["tex"], _v(m["color"]), _f(m["roughness"]), _f(m["ior"]),
            _f(m["intensity"]), m["two_sided"], _v(m["absorb"]), _f(m["wave_amp"]),
            _f(m["wave_freq"])))
    for m in state["meshes"]:
        lines.append("mesh %d %s %s" % (m["smooth"], path(m["file"]), m["usemtl"] or "-"))
    for o in state["objects"]:
        lines.append("object %d %d %d %d %d %d %s" % (o["kind"], o["mesh"], o["mat_front"],
                                                     o["mat_back"], o["cutout"], o["light"],
                                                     _v(o["xform"])))
    for l in state["lights"]:
        lines.append("light %d %s %s %s %s %s %s %s %s %d %d %d" % (
            l["kind"], _v(l["p"]), _v(l["u"]), _v(l["v"]), _v(l["n"]), _v(l["L"]),
            _f(l["radius"]), _f(l["area"]), _v(l["dir"]), l["two_sided"], l["tex"], l["flame"]))
    for f in state["flames"]:
        lines.append("flame %s %s %s %s %s %s %d %d" % (
            _v(f["base"]), _f(f["height"]), _f(f["radius"]), _f(f["intensity"]), _f(f["sigma"]),
            _f(f["noise_scale"]), f["seed"], f["steps"]))
    return "\n".join(lines) + "\n", r


class OracleScene(object):
    def __init__(self, text):
        lib = load()
        err = ctypes.create_string_buffer(512)
        self.h = lib.sdo_scene_load(text.encode(), err, 512)
        if not self.h:
            raise RuntimeError("oracle: " + err.value.decode())
        self.lib = lib

    def render(self, x0, y0, w, h, s0, s1, threads=1, film=None, aov=False):
        """Fold samples [s0, s1) of the rectangle into film (h, w, 4)."""
        if film is None:
            film = np.zeros((h, w, 4), np.float32)
        alb = np.zeros_like(film) if aov else None
        nrm = np.zeros_like(film) if aov else None
        rays = self.lib.sdo_render(self.h, x0, y0, w, h, s0, s1, threads, film.ctypes.data,
                                   alb.ctypes.data if aov else None,
                                   nrm.ctypes.data if aov else None)
        return film, int(rays), alb, nrm

    def table(self, which):
        n = self.lib.sdo_scene_table(self.h, which, None, 0)
        if n < 0:
            return None
        out = np.zeros(n, np.float32)
        self.lib.sdo_scene_table(self.h, which, out.ctypes.data, n)
        return out

    def close(self):
        if self.h:
            self.lib.sdo_scene_free(self.h)
            self.h = None

    def __del__(self):
        self.close()
