"""Seeded synthetic workloads.

  cornell()     Cornell-style box: five Lambert rects, an emissive rect light
                (radiance 17,12,4), a GGX metal sphere (roughness 0.3) and a
                smooth glass sphere (ior 1.5); 256x256, 16 spp, depth 8,
                seed 1, clamp 0.
  instancing()  1024 instances of a subdivision-4 icosphere (5120 tris,
                vertices displaced along the normal by seeded fBm, amplitude
                0.05), uniformly random rotations, per-axis scale U[0.5,2]^3,
                each with its own Lambert / GGX metal (roughness U[0.05,0.6])
                / plastic material; a 1024x512 float equirect sky (gradient
                plus a 0.5 degree sun disk of radiance 1e5) sampled by its 2D
                CDF; 1920x1080, 64 spp, depth 8, seed 1, clamp 0.
  volumes()     a procedural flame (64 march steps) with its embedded point
                lights; a water plane (ior 1.33, fBm wave normals, absorption
                0.4/0.1/0.05 per unit) over a sand floor holding a nested glass
                sphere (ior 1.5); five rough glass panels (roughness 0 ...
                0.6, flattened spheres so each is a closed medium); an
                emissive 2048-triangle mesh light sampled by area CDF;
                2560x1440, 256 spp.

The meshes and the environment map reach the renderer as .obj / .hdr files,
because the drop-in ABI only loads assets from files; write_assets() creates
them (deterministically) in a directory of the caller's choosing.
"""

import math
import os
import struct

import numpy as np

from .scene import Scene, rotate_x, rotate_y, rotate_z, scale, translate

# ---- value-noise fBm (numpy), used only to displace the icosphere ------------


def _hash_u32(x):
    x = (x * np.uint32(747796405) + np.uint32(2891336453)).astype(np.uint32)
    x = (((x >> ((x >> np.uint32(28)) + np.uint32(4))) ^ x) * np.uint32(277803737)).astype(np.uint32)
    return ((x >> np.uint32(22)) ^ x).astype(np.uint32)


def _lattice(ix, iy, iz, seed):
    h = (ix.astype(np.uint32) * np.uint32(73856093)) ^ (iy.astype(np.uint32) * np.uint32(19349663)) \
        ^ (iz.astype(np.uint32) * np.uint32(83492791)) ^ np.uint32(seed)
    return _hash_u32(h.astype(np.uint32)).astype(np.float64) / 4294967296.0


def _vnoise(p, seed):
    f = np.floor(p)
    i = f.astype(np.int64)
    t = p - f
    t = t * t * (3.0 - 2.0 * t)
    c = {}
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                c[dx, dy, dz] = _lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
    x00 = c[0, 0, 0] + (c[1, 0, 0] - c[0, 0, 0]) * t[:, 0]
    x10 = c[0, 1, 0] + (c[1, 1, 0] - c[0, 1, 0]) * t[:, 0]
    x01 = c[0, 0, 1] + (c[1, 0, 1] - c[0, 0, 1]) * t[:, 0]
    x11 = c[0, 1, 1] + (c[1, 1, 1] - c[0, 1, 1]) * t[:, 0]
    y0 = x00 + (x10 - x00) * t[:, 1]
    y1 = x01 + (x11 - x01) * t[:, 1]
    return y0 + (y1 - y0) * t[:, 2]


def fbm3(p, seed):
    amp, s = 0.5, np.zeros(len(p))
    for i in range(3):
        s += amp * _vnoise(p, (seed + i * 101) & 0xFFFFFFFF)
        p = 2.03 * p + np.array([11.7, 5.3, 7.9])
        amp *= 0.5
    return s


# ---- geometry -----------------------------------------------------------------


def icosphere(subdiv):
    """Unit icosphere by midpoint subdivision: 20 * 4^n faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(x, float) / np.linalg.norm(x) for x in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[k] = len(verts) - 1
            return cache[k]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int64)


def write_obj(path, verts, faces):
    with open(path, "w") as f:
        f.write("# generated by sundog_b200.workloads\n")
        for p in verts:
            f.write("v %.9g %.9g %.9g\n" % (p[0], p[1], p[2]))
        for a, b, c in faces:
            f.write("f %d %d %d\n" % (a + 1, b + 1, c + 1))


def write_hdr(path, rgb):
    """Radiance RGBE, flat scanlines, row 0 = top (-Y H +X W)."""
    h, w, _ = rgb.shape
    m = rgb.max(axis=2)
    e = np.zeros(m.shape, np.int32)
    mant = np.zeros(m.shape)
    nz = m > 1e-32
    mant[nz], e[nz] = np.frexp(m[nz])
    out = np.zeros((h, w, 4), np.uint8)
    sc = np.where(nz, mant * 256.0 / np.where(nz, m, 1.0), 0.0)
    for c in range(3):
        out[..., c] = np.clip(rgb[..., c] * sc, 0, 255).astype(np.uint8)
    out[..., 3] = np.where(nz, e + 128, 0).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(("-Y %d +X %d\n" % (h, w)).encode())
        f.write(out.tobytes())


def sky_image(w=1024, h=512, sun_elev_deg=35.0, sun_azim_deg=40.0, sun_radiance=1e5,
              sun_diam_deg=0.5):
    """Sky gradient (zenith blue to white horizon, dim ground) plus a sun disk."""
    rows = (np.arange(h) + 0.5) / h
    cols = (np.arange(w) + 0.5) / w
    theta = rows * math.pi
    phi = 2.0 * math.pi * cols - math.pi
    th, ph = np.meshgrid(theta, phi, indexing="ij")
    d = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], -1)
    up = np.clip(d[..., 1], 0.0, 1.0)[..., None]
    zen = np.array([0.25, 0.45, 0.95])
    hor = np.array([0.95, 0.95, 1.0])
    gnd = np.array([0.18, 0.16, 0.14])
    sky = hor + (zen - hor) * np.sqrt(up)
    img = np.where(d[..., 1:2] >= 0.0, sky, gnd)
    el, az = math.radians(sun_elev_deg), math.radians(sun_azim_deg)
    sd = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    cosang = np.clip(d @ sd, -1.0, 1.0)
    disk = cosang >= math.cos(math.radians(sun_diam_deg / 2.0))
    img[disk] = sun_radiance
    # Guarantee the sun covers at least the texel nearest to its centre.
    r = int(min(h - 1, math.acos(sd[1]) / math.pi * h))
    c = int(((math.atan2(sd[2], sd[0]) + math.pi) / (2 * math.pi) * w)) % w
    img[r, c] = sun_radiance
    return img.astype(np.float32)


def _uniform_rotation_euler(rng):
    """Uniform random rotation (Shoemake quaternion) as X, Y, Z degrees for
    steps applied in that order (R = Rz Ry Rx)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
                  math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3),
                  math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    ry = math.asin(-max(-1.0, min(1.0, R[2, 0])))
    rx = math.atan2(R[2, 1], R[2, 2])
    rz = math.atan2(R[1, 0], R[0, 0])
    return math.degrees(rx), math.degrees(ry), math.degrees(rz)


# ---- the workloads ------------------------------------------------------------------


def cornell(width=256, height=256, spp=16):
    s = Scene()
    s.render(width=width, height=height, spp=spp, max_depth=8, seed=1, clamp=0.0)
    s.camera(lookfrom=[0, 1, 3.9], lookat=[0, 1, 0], vfov=40)
    s.background_solid([0, 0, 0])
    s.lambert("grey", color=[0.73, 0.73, 0.73])
    s.lambert("red", color=[0.65, 0.05, 0.05])
    s.lambert("green", color=[0.12, 0.45, 0.15])
    s.emissive("lamp", color=[17, 12, 4], intensity=1.0)
    s.metal("metal", color=[0.9, 0.85, 0.8], roughness=0.3)
    s.dielectric("glass", ior=1.5)
    s.add("rect", "grey")                                            # floor
    s.add("rect", "grey", rotate_x(180), translate(0, 2, 0))         # ceiling
    s.add("rect", "grey", rotate_x(90), translate(0, 1, -1))         # back wall
    s.add("rect", "red", rotate_z(-90), translate(-1, 1, 0))         # left wall
    s.add("rect", "green", rotate_z(90), translate(1, 1, 0))         # right wall
    s.add("rect", "lamp", scale(0.25), rotate_x(180), translate(0, 1.99, 0))
    s.add("sphere", "metal", scale(0.35), translate(-0.42, 0.35, -0.3))
    s.add("sphere", "glass", scale(0.35), translate(0.42, 0.35, 0.3))
    return s


def write_instancing_assets(asset_dir, env_w=1024, env_h=512):
    os.makedirs(asset_dir, exist_ok=True)
    mesh = os.path.join(asset_dir, "icosphere4_fbm.obj")
    if not os.path.exists(mesh):
        v, f = icosphere(4)
        disp = 0.05 * (fbm3(v * 2.5, 1) - 0.4375)
        write_obj(mesh, v * (1.0 + disp)[:, None], f)
    env = os.path.join(asset_dir, "sky_%dx%d.hdr" % (env_w, env_h))
    if not os.path.exists(env):
        write_hdr(env, sky_image(env_w, env_h))
    return mesh, env


def instancing(asset_dir, width=1920, height=1080, spp=64, count=1024):
    mesh, env = write_instancing_assets(asset_dir)
    s = Scene()
    s.render(width=width, height=height, spp=spp, max_depth=8, seed=1, clamp=0.0)
    s.camera(lookfrom=[0, 22, 62], lookat=[0, 0, -4], vfov=45)
    s.background_envmap(os.path.basename(env), rotate=0, intensity=1.0, importance=True)
    s.mesh("ico", os.path.basename(mesh), normals="smooth")
    lay = np.random.default_rng(2)
    mats = np.random.default_rng(3)
    side = int(math.ceil(math.sqrt(count)))
    spacing = 4.2
    for k in range(count):
        i, j = k % side, k // side
        x = (i - (side - 1) / 2.0) * spacing + lay.uniform(-1.0, 1.0)
        z = (j - (side - 1) / 2.0) * spacing + lay.uniform(-1.0, 1.0)
        y = lay.uniform(0.0, 6.0)
        rx, ry, rz = _uniform_rotation_euler(lay)
        sc = lay.uniform(0.5, 2.0, 3)
        kind = int(mats.integers(0, 3))
        name = "m%04d" % k
        if kind == 0:
            s.lambert(name, color=list(mats.uniform(0.15, 0.9, 3)))
        elif kind == 1:
            s.metal(name, color=list(mats.uniform(0.5, 1.0, 3)),
                    roughness=float(mats.uniform(0.05, 0.6)))
        else:
            s.plastic(name, color=list(mats.uniform(0.1, 0.9, 3)),
                      roughness=float(mats.uniform(0.05, 0.4)))
        s.add("mesh:ico", name, scale(*sc), rotate_x(rx), rotate_y(ry), rotate_z(rz),
              translate(x, y, z))
    return s


def light_canopy(n=32, size=2.4, seed=4):
    """An n x n grid (2 n^2 triangles) gently warped by seeded noise."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-size, size, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    Y = 0.08 * np.sin(1.7 * X) * np.cos(1.3 * Z) + 0.02 * rng.standard_normal(X.shape)
    verts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1)
    faces = []
    for i in range(n):
        for j in range(n):
            a = i * (n + 1) + j
            b, c, d = a + 1, a + n + 1, a + n + 2
            faces += [(a, b, d), (a, d, c)]
    return verts, np.array(faces)


def write_volume_assets(asset_dir):
    os.makedirs(asset_dir, exist_ok=True)
    mesh = os.path.join(asset_dir, "canopy_2048.obj")
    if not os.path.exists(mesh):
        v, f = light_canopy()
        write_obj(mesh, v, f)
    return mesh


def volumes(asset_dir, width=2560, height=1440, spp=256, flame_steps=64):
    mesh = write_volume_assets(asset_dir)
    s = Scene()
    s.render(width=width, height=height, spp=spp, max_depth=8, seed=1, clamp=0.0)
    s.camera(lookfrom=[0, 3.2, 9.5], lookat=[0, 0.6, 0], vfov=42)
    s.background_gradient(horizon=[0.03, 0.035, 0.05], zenith=[0.005, 0.008, 0.02])
    s.water("water", ior=1.33, absorb=[0.4, 0.1, 0.05], wave_amp=0.06, wave_freq=2.0)
    s.lambert("sand", color=[0.7, 0.6, 0.45])
    s.lambert("stone", color=[0.35, 0.33, 0.3])
    s.dielectric("glass", ior=1.5)
    for k, r in enumerate([0.0, 0.15, 0.3, 0.45, 0.6]):
        s.dielectric("panel%d" % k, ior=1.5, roughness=r)
    s.emissive("canopy", color=[1.0, 0.9, 0.75], intensity=6.0, two_sided=False)
    s.mesh("canopy", os.path.basename(mesh), normals="flat")
    s.add("rect", "sand", scale(8), translate(0, -1.2, 0))                # pool floor
    s.add("rect", "water", scale(8))                                     # water surface
    s.add("sphere", "glass", scale(0.8), translate(0.6, -0.2, 0.8))      # nested in water
    s.add("cylinder", "stone", scale(0.7, 0.25, 0.7), translate(-2.6, 0.25, -0.5))
    s.add("disk", "stone", scale(0.7), translate(-2.6, 0.5, -0.5))
    for k in range(5):
        x = -3.2 + 1.6 * k
        s.add("sphere", "panel%d" % k, scale(0.55, 0.8, 0.06), rotate_y(-20 + 10 * k),
              translate(x, 1.3, -2.4))
    s.add("mesh:canopy", "canopy", rotate_x(180), translate(0, 4.2, -0.5))
    s.flame(base=[-2.6, 0.5, -0.5], height=1.4, radius=0.45, intensity=20.0, sigma=4.0,
            noise_scale=3.0, seed=3, light_intensity=12.0, steps=flame_steps)
    return s


def write_ppm(path, rgb8):
    """Binary PPM (P6), row 0 = top."""
    h, w, _ = rgb8.shape
    with open(path, "wb") as f:
        f.write(("P6\n%d %d\n255\n" % (w, h)).encode())
        f.write(np.ascontiguousarray(rgb8, np.uint8).tobytes())


def write_pam(path, rgba8):
    """Binary PAM (P7) with an alpha channel, row 0 = top."""
    h, w, _ = rgba8.shape
    with open(path, "wb") as f:
        f.write(("P7\nWIDTH %d\nHEIGHT %d\nDEPTH 4\nMAXVAL 255\nTUPLTYPE RGB_ALPHA\nENDHDR\n"
                 % (w, h)).encode())
        f.write(np.ascontiguousarray(rgba8, np.uint8).tobytes())


def write_textured_assets(asset_dir):
    """Images and a uv-mapped mesh for the textured scene: a 96x64 sRGB
    colour ramp with a seeded speckle, a 40x40 linear (non-sRGB) stripe
    image, a 64x64 RGBA leaf mask (alpha 0 outside a lobed outline and in
    round holes) and a 4x4-quad uv grid mesh."""
    os.makedirs(asset_dir, exist_ok=True)
    ramp = os.path.join(asset_dir, "tex_ramp.ppm")
    if not os.path.exists(ramp):
        rng = np.random.default_rng(11)
        y, x = np.mgrid[0:64, 0:96]
        img = np.stack([x * 255 / 95, y * 255 / 63, 128 + 100 * np.sin(x * 0.3) * np.cos(y * 0.2)], -1)
        img = np.clip(img + rng.integers(-20, 21, img.shape), 0, 255)
        write_ppm(ramp, img.astype(np.uint8))
    stripes = os.path.join(asset_dir, "tex_stripes.ppm")
    if not os.path.exists(stripes):
        y, x = np.mgrid[0:40, 0:40]
        band = ((x + y) // 5) % 2
        img = np.stack([200 * band + 30, 60 + 0 * x, 220 - 180 * band], -1)
        write_ppm(stripes, img.astype(np.uint8))
    leaf = os.path.join(asset_dir, "tex_leaf.pam")
    if not os.path.exists(leaf):
        y, x = np.mgrid[0:64, 0:64]
        u, v = (x - 31.5) / 32.0, (y - 31.5) / 32.0
        r, a = np.hypot(u, v), np.arctan2(v, u)
        inside = r < 0.75 + 0.2 * np.cos(5 * a)
        holes = np.hypot(u - 0.25, v + 0.1) < 0.12
        holes |= np.hypot(u + 0.3, v - 0.3) < 0.1
        alpha = np.where(inside & ~holes, 255, 0)
        img = np.stack([40 + 60 * (u + 1), 150 + 40 * v, 50 + 0 * u, alpha], -1)
        write_pam(leaf, np.clip(img, 0, 255).astype(np.uint8))
    grid = os.path.join(asset_dir, "uv_grid.obj")
    if not os.path.exists(grid):
        n = 4
        with open(grid, "w") as f:
            f.write("# generated by sundog_b200.workloads: %dx%d quads with uv\n" % (n, n))
            for j in range(n + 1):
                for i in range(n + 1):
                    f.write("v %.6f %.6f 0\n" % (i / n - 0.5, j / n - 0.5))
                    f.write("vt %.6f %.6f\n" % (i / n, j / n))
            for j in range(n):
                for i in range(n):
                    a = j * (n + 1) + i + 1
                    b, c, d = a + 1, a + n + 1, a + n + 2
                    f.write("f %d/%d %d/%d %d/%d\n" % (a, a, b, b, d, d))
                    f.write("f %d/%d %d/%d %d/%d\n" % (a, a, d, d, c, c))
    return ramp, stripes, leaf, grid


def textured(asset_dir, width=96, height=64, spp=16):
    """Image textures and alpha cutouts: an sRGB image on the floor, a linear
    image on a sphere, an image-textured emissive rect (textured NEE light),
    a cutout leaf on a rect and on a uv-mapped triangle mesh in front of a
    point light (cutout shadows), and a glass sphere."""
    ramp, stripes, leaf, grid = write_textured_assets(asset_dir)
    s = Scene()
    s.render(width=width, height=height, spp=spp, max_depth=8, seed=5, clamp=0.0)
    s.camera(lookfrom=[0, 2.2, 6.5], lookat=[0, 0.8, 0], vfov=42)
    s.background_gradient(horizon=[0.6, 0.65, 0.7], zenith=[0.2, 0.3, 0.5])
    s.texture("ramp", "image", file=os.path.basename(ramp))
    s.texture("stripes", "image", file=os.path.basename(stripes), srgb=False)
    s.texture("leafmask", "image", file=os.path.basename(leaf))
    s.lambert("floor", texture="ramp")
    s.lambert("striped", texture="stripes")
    s.lambert("leaf", texture="leafmask")
    s.plastic("leafgloss", texture="leafmask", roughness=0.3)
    s.emissive("sign", texture="ramp", intensity=4.0)
    s.dielectric("glass", ior=1.5)
    s.mesh("grid", os.path.basename(grid), normals="flat")
    s.point_light(position=[1.5, 4.0, 2.5], intensity=[40, 38, 34], radius=0.2)
    s.add("rect", "floor", scale(5))
    s.add("sphere", "striped", scale(0.7), rotate_y(25), translate(-1.6, 0.7, 0.2))
    s.add("sphere", "glass", scale(0.5), translate(1.7, 0.5, 0.9))
    s.add("rect", "sign", scale(1.0, 1, 0.5), rotate_x(90), translate(1.6, 1.4, -2.0))
    s.add("rect", "leaf", scale(0.9), rotate_x(70), translate(0.4, 1.5, 1.2),
          cutout="leafmask")
    s.add("mesh:grid", "leafgloss", scale(1.6), rotate_y(-30), translate(-0.5, 1.1, -0.6),
          material_back="leaf", cutout="leafmask")
    return s

CONFIGS = {
    0: ("cornell", "Plain NEE+MIS Cornell box 256x256 16spp depth 8 seed 1"),
    1: ("instancing", "1024 icosphere-4 instances + 1024x512 env, 1920x1080 64spp"),
    2: ("volumes", "flame + water + nested glass + rough panels + 2048-tri mesh light, "
                   "2560x1440 256spp"),
}


def features():
    """Feature coverage at 72x48, 8 spp: every quadric kind, checker and grid
    textures, Lambert / metal / glass / rough glass / plastic / water
    materials, an emissive rect (auto NEE), a soft point light, a distant
    light, a thin-lens camera and a gradient sky."""
    s = Scene()
    s.render(width=72, height=48, spp=8, max_depth=8, seed=3, clamp=0.0)
    s.camera(lookfrom=[0, 3.0, 8.5], lookat=[0, 0.9, 0], vfov=40, aperture=0.03)
    s.background_gradient(horizon=[0.9, 0.9, 0.95], zenith=[0.35, 0.55, 0.95])
    s.texture("floor", "checker", a=[0.8, 0.8, 0.8], b=[0.25, 0.25, 0.3], scale=[12, 12])
    s.texture("lines", "grid", a=[0.7, 0.6, 0.5], b=[0.1, 0.1, 0.1], scale=[6, 6], width=0.08)
    s.lambert("ground", texture="floor")
    s.lambert("red", color=[0.75, 0.25, 0.25])
    s.lambert("gridded", texture="lines")
    s.metal("gold", color=[1.0, 0.78, 0.34], roughness=0.15)
    s.metal("mirror", color=[0.9, 0.9, 0.9], roughness=0.0)
    s.dielectric("glass", ior=1.5)
    s.dielectric("frost", ior=1.45, roughness=0.3, absorb=[0.1, 0.2, 0.3])
    s.plastic("toy", color=[0.2, 0.5, 0.8], roughness=0.2)
    s.water("pool", absorb=[0.3, 0.1, 0.05])
    s.emissive("lamp", color=[1.0, 0.95, 0.85], intensity=20.0)
    s.point_light(position=[5, 5, 4], intensity=[30, 30, 30], radius=0.3)
    s.distant_light(direction=[-0.5, -1, -0.3], radiance=[0.6, 0.6, 0.55])
    s.add("rect", "ground", scale(8))
    s.add("sphere", "glass", scale(0.8), translate(-3.0, 0.8, 1.0))
    s.add("sphere", "red", scale(0.8), translate(-1.0, 0.8, 1.0))
    s.add("cylinder", "gold", scale(0.6, 0.8, 0.6), translate(1.0, 0.8, 1.0))
    s.add("parabola", "mirror", scale(1.4, 1.4, 1.4), rotate_z(90), translate(3.4, 1.4, 0.0),
          material_back=None)
    s.add("disk", "mirror", scale(1.6), rotate_x(90), translate(0, 1.6, -3.2))
    s.add("rect", "lamp", rotate_x(180), scale(1.2), translate(0, 6, 2))
    s.add("sphere", "frost", scale(0.5, 0.7, 0.5), translate(2.2, 0.7, 2.4))
    s.add("sphere", "toy", scale(0.45), rotate_y(30), translate(-2.0, 0.45, 2.6))
    s.add("rect", "gridded", scale(1.0, 1, 0.6), rotate_x(70), translate(-3.5, 1.0, -2.0))
    s.add("rect", "pool", scale(1.2), translate(0.2, 0.05, 3.2))
    return s


def make(config, asset_dir, **kw):
    if config == 0:
        return cornell(**kw)
    if config == 1:
        return instancing(asset_dir, **kw)
    if config == 2:
        return volumes(asset_dir, **kw)
    raise ValueError("unknown config %r" % config)
