"""Python scene builder over libsundog.so.

Mirrors the method names and argument meaning of sundog's scene library
(scenes/scenelib.py: Scene.render/camera/background_*/texture/material/
lambert/metal/dielectric/emissive/water/plastic/mesh/add/point_light/
distant_light/flame/physics, and the scale/rotate_*/translate steps) so that
scene descriptions and tests read the same. Arguments left unset are not
sent, and the renderer's own defaults apply. Registry ids are allocated by
sorted name, as scenelib does (scenes/scenelib.py:538-540), and calls are
replayed in the ABI's phase order: config, registries, objects, flames,
explicit lights.

Beyond scenelib: flame(steps=N) sets the ray-march step count, and the
render helpers return the film as numpy arrays through sundog_render_ex or a
resident session.
"""

import ctypes
import math

import numpy as np

from . import abi

NAN = float("nan")
GEOM = {"sphere": 0, "rect": 1, "disk": 2, "cylinder": 3, "parabola": 4}


class SceneError(ValueError):
    """A scene call was rejected; the message is the library's."""


def scale(x, y=None, z=None):
    if y is None and z is None:
        if isinstance(x, (list, tuple)):
            return ("scale", tuple(float(v) for v in x))
        return ("scale", (float(x),) * 3)
    return ("scale", (float(x), float(y), float(z)))


def translate(x, y=None, z=None):
    if y is None and z is None:
        return ("translate", tuple(float(v) for v in x))
    return ("translate", (float(x), float(y), float(z)))


def rotate_x(deg):
    return ("rotate_x", (float(deg), 0.0, 0.0))


def rotate_y(deg):
    return ("rotate_y", (float(deg), 0.0, 0.0))


def rotate_z(deg):
    return ("rotate_z", (float(deg), 0.0, 0.0))


_STEP_KIND = {"scale": 0, "translate": 1, "rotate_x": 2, "rotate_y": 3, "rotate_z": 4}


def _d3(v):
    return abi.c_d3(*[float(c) for c in v]) if v is not None else None


def _f(v):
    return NAN if v is None else float(v)


def _tri(v):
    return -1 if v is None else (1 if v else 0)


class Scene(object):
    def __init__(self):
        self._render = {}
        self._camera = None
        self._background = None
        self._physics = None
        self._textures = {}
        self._materials = {}
        self._meshes = {}
        self._objects = []
        self._flames = []
        self._lights = []

    # ---- configuration ---------------------------------------------------------
    def render(self, width=None, height=None, spp=None, max_depth=None, clamp=None, seed=None,
               exposure=None, transparent_shadows=None):
        for k, v in dict(width=width, height=height, spp=spp, max_depth=max_depth, clamp=clamp,
                         seed=seed, exposure=exposure,
                         transparent_shadows=transparent_shadows).items():
            if v is not None:
                self._render[k] = v

    def camera(self, lookfrom, lookat, up=None, vfov=None, aperture=None, focus_dist=None):
        self._camera = (lookfrom, lookat, up, vfov, aperture, focus_dist)

    def background_solid(self, color):
        self._background = ("solid", color)

    def background_gradient(self, horizon, zenith):
        self._background = ("gradient", horizon, zenith)

    def background_envmap(self, file, rotate=None, intensity=None, importance=None):
        self._background = ("envmap", file, rotate, intensity, importance)

    def physics(self, gravity=None, timestep=None, max_time=None, friction=None, restitution=None,
                solver_iterations=None, sleep_threshold=None, stop_time=None):
        self._physics = (gravity, timestep, max_time, friction, restitution, solver_iterations,
                         sleep_threshold, stop_time)

    # ---- registries ----------------------------------------------------------------
    def texture(self, name, type, **f):
        self._textures[name] = (type, f)
        return name

    def material(self, name, type, **f):
        self._materials[name] = (type, {k: v for k, v in f.items() if v is not None})
        return name

    def lambert(self, name, color=None, texture=None):
        return self.material(name, "lambert", color=color, texture=texture)

    def metal(self, name, color=None, texture=None, roughness=None):
        return self.material(name, "metal", color=color, texture=texture, roughness=roughness)

    def dielectric(self, name, ior=None, absorb=None, roughness=None):
        return self.material(name, "dielectric", ior=ior, absorb=absorb, roughness=roughness)

    def emissive(self, name, color=None, texture=None, intensity=None, two_sided=None):
        return self.material(name, "emissive", color=color, texture=texture,
                             intensity=intensity, two_sided=two_sided)

    def water(self, name, ior=None, absorb=None, wave_amp=None, wave_freq=None):
        return self.material(name, "water", ior=ior, absorb=absorb, wave_amp=wave_amp,
                             wave_freq=wave_freq)

    def plastic(self, name, color=None, texture=None, roughness=None):
        return self.material(name, "plastic", color=color, texture=texture, roughness=roughness)

    def mesh(self, name, obj, normals=None, usemtl=None):
        self._meshes[name] = (obj, normals, usemtl)
        return "mesh:" + name

    # ---- objects / lights ---------------------------------------------------------
    def add(self, shape, material, *steps, material_back="__same__", cutout=None, nee=None,
            physics=None):
        self._objects.append((shape, material, list(steps), material_back, cutout, nee, physics))

    def flame(self, base, height, radius, intensity=None, sigma=None, noise_scale=None, seed=None,
              light_intensity=None, steps=None):
        self._flames.append((base, height, radius, intensity, sigma, noise_scale, seed,
                             light_intensity, steps))

    def point_light(self, position, intensity, radius=None):
        self._lights.append(("point", position, intensity, radius))

    def distant_light(self, direction, radiance):
        self._lights.append(("distant", direction, radiance))

    # ---- replay against the library ---------------------------------------------
    def build(self, base_dir=".", lib=None):
        """Create a sundog_scene handle and replay every call; returns the handle."""
        lib = lib or abi.load()
        tex_ids = {n: i for i, n in enumerate(sorted(self._textures))}
        mat_ids = {n: i for i, n in enumerate(sorted(self._materials))}
        mesh_ids = {n: i for i, n in enumerate(sorted(self._meshes))}
        h = lib.sundog_scene_create(base_dir.encode())
        if not h:
            raise SceneError(abi.last_error(lib))
        try:
            self._replay(lib, h, tex_ids, mat_ids, mesh_ids)
        except Exception:
            lib.sundog_scene_destroy(h)
            raise
        return h

    def _replay(self, lib, h, tex_ids, mat_ids, mesh_ids):
        def ok(rc, what, setter=False):
            if rc is None or rc < 0 or (setter and rc != 0):
                raise SceneError("%s: %s" % (what, abi.last_error(lib)))
            return rc

        r = self._render
        ts = r.get("transparent_shadows")
        ok(lib.sundog_set_render(h, int(r.get("width", -1)), int(r.get("height", -1)),
                                 int(r.get("spp", -1)), int(r.get("max_depth", -1)),
                                 _f(r.get("clamp")), int(r.get("seed", -1)),
                                 _f(r.get("exposure")), _tri(ts)), "render", True)
        if self._physics is not None:
            g, tstep, mt, fr, re, si, sl, st = self._physics
            ok(lib.sundog_set_physics(h, _d3(g), _f(tstep), _f(mt), _f(fr), _f(re),
                                      int(si[0]) if si else -1, int(si[1]) if si else -1,
                                      _f(sl), _f(st)), "physics", True)
        if self._camera is not None:
            lf, la, up, vf, ap, fd = self._camera
            ok(lib.sundog_set_camera(h, _d3(lf), _d3(la), _d3(up), _f(vf), _f(ap), _f(fd)),
               "camera", True)
        b = self._background
        if b is not None:
            if b[0] == "solid":
                ok(lib.sundog_set_background_solid(h, _d3(b[1])), "background", True)
            elif b[0] == "gradient":
                ok(lib.sundog_set_background_gradient(h, _d3(b[1]), _d3(b[2])), "background",
                   True)
            else:
                ok(lib.sundog_set_background_envmap(h, b[1].encode(), _f(b[2]), _f(b[3]),
                                                    _tri(b[4])), "envmap", True)
        for name in sorted(self._textures):
            kind, f = self._textures[name]
            sc = f.get("scale")
            sc2 = (ctypes.c_double * 2)(*sc) if sc is not None else None
            if kind == "solid":
                rc = lib.sundog_add_texture_solid(h, _d3(f["color"]))
            elif kind == "checker":
                rc = lib.sundog_add_texture_checker(h, _d3(f["a"]), _d3(f["b"]), sc2)
            elif kind == "grid":
                rc = lib.sundog_add_texture_grid(h, _d3(f["a"]), _d3(f["b"]), sc2,
                                                 _f(f.get("width")))
            else:
                rc = lib.sundog_add_texture_image(h, f["file"].encode(), _tri(f.get("srgb")))
            ok(rc, "texture %r" % name)
        for name in sorted(self._materials):
            kind, f = self._materials[name]
            tid = tex_ids[f["texture"]] if "texture" in f else -1
            col = _d3(f.get("color"))
            if kind == "lambert":
                rc = lib.sundog_add_material_lambert(h, col, tid)
            elif kind == "metal":
                rc = lib.sundog_add_material_metal(h, col, tid, _f(f.get("roughness")))
            elif kind == "dielectric":
                rc = lib.sundog_add_material_dielectric(h, _f(f.get("ior")), _d3(f.get("absorb")),
                                                        col, tid, _f(f.get("roughness")))
            elif kind == "emissive":
                rc = lib.sundog_add_material_emissive(h, col, tid, _f(f.get("intensity")),
                                                      _tri(f.get("two_sided")))
            elif kind == "water":
                rc = lib.sundog_add_material_water(h, _f(f.get("ior")), _d3(f.get("absorb")),
                                                   _f(f.get("wave_amp")), _f(f.get("wave_freq")),
                                                   col)
            elif kind == "plastic":
                rc = lib.sundog_add_material_plastic(h, col, tid, _f(f.get("roughness")))
            else:
                raise SceneError("material %r: unknown type %r" % (name, kind))
            ok(rc, "material %r" % name)
        for name in sorted(self._meshes):
            obj, normals, usemtl = self._meshes[name]
            smooth = -1 if normals is None else (1 if normals == "smooth" else 0)
            ok(lib.sundog_add_mesh(h, obj.encode(), smooth, usemtl.encode() if usemtl else None),
               "mesh %r" % name)
        for shape, mat, steps, back, cutout, nee, phys in self._objects:
            if shape.startswith("mesh:"):
                gk, mid = 5, mesh_ids[shape[5:]]
            else:
                gk, mid = GEOM[shape], -1
            front = -1 if mat is None else mat_ids[mat]
            if back == "__same__":
                bk = -2
            elif back is None:
                bk = -1
            else:
                bk = mat_ids[back]
            arr = (abi.XformStep * max(len(steps), 1))()
            for i, (k, v) in enumerate(steps):
                arr[i] = abi.XformStep(_STEP_KIND[k], v[0], v[1], v[2])
            pb = None
            if phys is not None:
                pb = abi.PhysicsBody(1 if phys.get("dynamic") else 0, _f(phys.get("density")),
                                     1 if "velocity" in phys else 0,
                                     1 if "angular_velocity" in phys else 0,
                                     abi.c_d3(*phys.get("velocity", (0, 0, 0))),
                                     abi.c_d3(*phys.get("angular_velocity", (0, 0, 0))),
                                     _f(phys.get("friction")), _f(phys.get("restitution")),
                                     _f(phys.get("thickness")))
            ok(lib.sundog_add_object(h, gk, mid, front, bk,
                                     tex_ids[cutout] if cutout is not None else -1, arr,
                                     len(steps), _tri(nee), ctypes.byref(pb) if pb else None),
               "object %s" % shape)
        for base, ht, rad, inten, sig, ns, seed, li, steps in self._flames:
            fid = ok(lib.sundog_add_flame(h, _d3(base), float(ht), float(rad), _f(inten), _f(sig),
                                          _f(ns), int(seed) if seed is not None else -1, _f(li)),
                     "flame")
            if steps is not None:
                ok(lib.sundog_set_flame_steps(h, fid, int(steps)), "flame steps", True)
        for l in self._lights:
            if l[0] == "point":
                rc = lib.sundog_add_point_light(h, _d3(l[1]), _d3(l[2]), _f(l[3]))
            else:
                rc = lib.sundog_add_distant_light(h, _d3(l[1]), _d3(l[2]))
            ok(rc, "light")

    # ---- rendering ----------------------------------------------------------------
    def render_film(self, base_dir=".", aov=False, chunk_spp=0, engine=0, **opts):
        """Render through sundog_render_ex; returns (film HxWx4, result, aovs)."""
        lib = abi.load()
        h = self.build(base_dir, lib)
        try:
            o = abi.options(**opts)
            w = opts.get("width", -1)
            w = w if w > 0 else int(self._render.get("width", 1280))
            ht = opts.get("height", -1)
            ht = ht if ht > 0 else int(self._render.get("height", 720))
            film = np.zeros((ht, w, 4), np.float32)
            alb = np.zeros_like(film) if aov else None
            nrm = np.zeros_like(film) if aov else None
            ext = abi.RenderExt(film.ctypes.data, alb.ctypes.data if aov else None,
                                nrm.ctypes.data if aov else None, chunk_spp, 1, 0, 0, 0,
                                engine)
            res = abi.RenderResult()
            abi.check(lib.sundog_render_ex(h, ctypes.byref(o), ctypes.byref(ext),
                                           ctypes.byref(res)), "render", lib)
            return film, res, (alb, nrm)
        finally:
            lib.sundog_scene_destroy(h)


class Session(object):
    """A scene resident on the device (sundog_session_*)."""

    def __init__(self, scene, base_dir=".", aov=False, chunk_spp=0, guiding=0, sample_offset=0,
                 frame_spp=0, engine=0, shard_count=0, shard_index=0, **opts):
        self.lib = abi.load()
        h = scene.build(base_dir, self.lib)
        try:
            o = abi.options(**opts)
            dummy = np.zeros(4, np.float32)
            ext = abi.RenderExt(None, dummy.ctypes.data if aov else None, None, chunk_spp, 1,
                                guiding, sample_offset, frame_spp, engine, shard_count,
                                shard_index)
            self.handle = self.lib.sundog_session_create(h, ctypes.byref(o), ctypes.byref(ext))
            if not self.handle:
                raise abi.SundogError("session: " + abi.last_error(self.lib))
        finally:
            self.lib.sundog_scene_destroy(h)
        self.aov = aov
        self.stats = abi.SessionStats()
        abi.check(self.lib.sundog_session_info(self.handle, ctypes.byref(self.stats)), "info",
                  self.lib)

    def render(self, stream=None, reset=True):
        """One full render on `stream` (a cudaStream_t as int; None = own)."""
        res = abi.RenderResult()
        abi.check(self.lib.sundog_session_render(self.handle, stream, 1 if reset else 0,
                                                 ctypes.byref(res)), "session render", self.lib)
        return res

    def set_guiding(self, enable=True, **cfg):
        """Learned path guiding for later renders; cfg overrides defaults
        (train_spp, pass_spp, steps_per_pass, batch, learning_rate, mix, seed,
        record_cap)."""
        c = abi.GuidingConfig()
        self.lib.sundog_guiding_defaults(ctypes.byref(c))
        for k, v in cfg.items():
            if not hasattr(c, k):
                raise TypeError("unknown guiding option %r" % k)
            setattr(c, k, v)
        abi.check(self.lib.sundog_session_set_guiding(self.handle, 1 if enable else 0,
                                                      ctypes.byref(c)), "guiding", self.lib)

    def guiding_stats(self):
        st = abi.GuidingStats()
        abi.check(self.lib.sundog_session_guiding_stats(self.handle, ctypes.byref(st)),
                  "guiding stats", self.lib)
        return st

    def guide_params(self):
        p = np.zeros(abi.GUIDE_PARAMS, np.float32)
        abi.check(self.lib.sundog_session_guide_params(self.handle, p.ctypes.data), "guide params",
                  self.lib)
        return p

    def guide_records(self, max_records=1 << 20):
        n = ctypes.c_uint64(0)
        abi.check(self.lib.sundog_session_guide_records(self.handle, None, 0, ctypes.byref(n)),
                  "guide records", self.lib)
        m = min(n.value, max_records)
        out = np.zeros((m, 12), np.float32)
        abi.check(self.lib.sundog_session_guide_records(self.handle, out.ctypes.data, m,
                                                        ctypes.byref(n)), "guide records",
                  self.lib)
        return out

    def read(self):
        s = self.stats
        film = np.zeros((s.height, s.width, 4), np.float32)
        if self.aov:
            alb = np.zeros_like(film)
            nrm = np.zeros_like(film)
            abi.check(self.lib.sundog_session_read(self.handle, film.ctypes.data, alb.ctypes.data,
                                                   nrm.ctypes.data), "read", self.lib)
            return film, alb, nrm
        abi.check(self.lib.sundog_session_read(self.handle, film.ctypes.data, None, None), "read",
                  self.lib)
        return film

    def denoise(self):
        """The film denoised on the device (needs a session created with
        aov=True): height x width x 4 float32."""
        s = self.stats
        out = np.zeros((s.height, s.width, 4), np.float32)
        abi.check(self.lib.sundog_session_denoise(self.handle, out.ctypes.data), "denoise",
                  self.lib)
        return out

    def copy_film(self, film_device_ptr, stream=None):
        """Device-to-device copy of the film into caller-owned device memory
        (width*height float4) on `stream` (a cudaStream_t as int)."""
        abi.check(self.lib.sundog_session_copy_film(self.handle, film_device_ptr, stream),
                  "copy film", self.lib)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.sundog_session_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()


def debug_json(handle, lib=None):
    import json
    lib = lib or abi.load()
    need = ctypes.c_size_t(0)
    abi.check(lib.sundog_scene_debug_json(handle, None, 0, ctypes.byref(need)), "debug", lib)
    buf = ctypes.create_string_buffer(need.value)
    abi.check(lib.sundog_scene_debug_json(handle, buf, need.value, ctypes.byref(need)), "debug",
              lib)
    return json.loads(buf.value.decode())
