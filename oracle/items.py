"""ORACLE — test infrastructure only (the checker, never the product).

numpy layouts of the function-vector items shared by the device self-test
(sundog_b200/csrc/selftest.cu), the oracle harness (oracle/fnvec.cpp) and the
golden vectors (tests/golden/), plus seeded input generators.
"""

import numpy as np

V3 = ("<f4", 3)

MAT = np.dtype([("kind", "<i4"), ("texId", "<i4"), ("color", V3), ("roughness", "<f4"),
                ("ior", "<f4"), ("intensity", "<f4"), ("twoSided", "<i4"), ("absorb", V3),
                ("waveAmp", "<f4"), ("waveFreq", "<f4")], align=True)
LIGHT = np.dtype([("kind", "<i4"), ("p", V3), ("u", V3), ("v", V3), ("n", V3), ("L", V3),
                  ("radius", "<f4"), ("area", "<f4"), ("dir", V3), ("twoSided", "<i4"),
                  ("texId", "<i4"), ("flameId", "<i4"), ("ptr", "<u8", 4), ("numTris", "<i4"),
                  ("ngSign", "<f4")], align=True)
FLAME = np.dtype([("base", V3), ("height", "<f4"), ("radius", "<f4"), ("intensity", "<f4"),
                  ("sigma", "<f4"), ("noiseScale", "<f4"), ("seed", "<u4"), ("steps", "<i4")],
                 align=True)

ITEMS = {
    # id: (name, input dtype, output dtype)
    1: ("pcg", np.dtype([("seed", "<u8"), ("seq", "<u8")], align=True),
        np.dtype([("next", "<u4", 8), ("uni", "<f4", 4)], align=True)),
    2: ("bsdf_eval", np.dtype([("m", MAT), ("albedo", V3), ("wo", V3), ("wi", V3), ("n", V3),
                               ("eta", "<f4")], align=True),
        np.dtype([("f", V3), ("pdf", "<f4")], align=True)),
    3: ("bsdf_draw", np.dtype([("m", MAT), ("albedo", V3), ("d", V3), ("n", V3), ("front", "<i4"),
                               ("etaExt", "<f4"), ("state", "<u8"), ("inc", "<u8")], align=True),
        np.dtype([("wi", V3), ("weight", V3), ("pdf", "<f4"), ("delta", "<i4"), ("ok", "<i4"),
                  ("pad", "<u4"), ("state", "<u8")], align=True)),
    4: ("quadric", np.dtype([("kind", "<i4"), ("o", V3), ("d", V3), ("tmin", "<f4"),
                             ("tmax", "<f4")], align=True),
        np.dtype([("count", "<i4"), ("t0", "<f4"), ("n0", V3), ("u0", "<f4"), ("v0", "<f4"),
                  ("t1", "<f4"), ("n1", V3), ("u1", "<f4"), ("v1", "<f4")], align=True)),
    5: ("triangle", np.dtype([("o", V3), ("d", V3), ("p0", V3), ("p1", V3), ("p2", V3),
                              ("tmin", "<f4"), ("tmax", "<f4")], align=True),
        np.dtype([("hit", "<i4"), ("t", "<f4"), ("b1", "<f4"), ("b2", "<f4")], align=True)),
    6: ("light", np.dtype([("l", LIGHT), ("x", V3), ("state", "<u8"), ("inc", "<u8")], align=True),
        np.dtype([("wi", V3), ("Li", V3), ("dist", "<f4"), ("pdf", "<f4"), ("delta", "<i4"),
                  ("ok", "<i4"), ("state", "<u8"), ("density", "<f4"), ("pad", "<f4")],
                 align=True)),
    7: ("flame", np.dtype([("f", FLAME), ("o", V3), ("d", V3), ("tEnd", "<f4"), ("skip", "<i4"),
                           ("state", "<u8"), ("inc", "<u8")], align=True),
        np.dtype([("Lv", V3), ("trans", V3), ("tr", "<f4"), ("pad", "<i4"),
                  ("stateMarch", "<u8"), ("stateShadow", "<u8")], align=True)),
    8: ("noise", np.dtype([("p", V3), ("seed", "<u4"), ("ns", V3), ("wo", V3), ("amp", "<f4"),
                           ("freq", "<f4")], align=True),
        np.dtype([("fbm", "<f4"), ("vnoise", "<f4"), ("wave", V3)], align=True)),
    9: ("cdf_search", np.dtype([("u", "<f4")]), np.dtype([("index", "<i4")])),
}

SIZES = {1: (16, 48), 2: (108, 16), 3: (120, 48), 4: (36, 52), 5: (68, 16), 6: (168, 56),
         7: (88, 48), 8: (48, 20), 9: (4, 4)}
for _k, (_n, _i, _o) in ITEMS.items():
    assert (_i.itemsize, _o.itemsize) == SIZES[_k], (_n, _i.itemsize, _o.itemsize)


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _hemi(rng, nrm, sign):
    v = _unit(rng, len(nrm))
    d = np.sum(v * nrm, axis=1, keepdims=True)
    return np.where(d * sign < 0, -v, v).astype(np.float32)


def random_materials(rng, n):
    m = np.zeros(n, MAT)
    kinds = rng.integers(0, 8, n)
    # 0 lambert, 1 metal mirror, 2 metal rough, 3 glass smooth, 4 glass rough,
    # 5 plastic, 6 water, 7 emissive
    kind_map = np.array([0, 1, 1, 2, 2, 5, 4, 3])
    m["kind"] = kind_map[kinds]
    m["texId"] = -1
    m["color"] = rng.uniform(0.05, 1.0, (n, 3))
    rough = rng.uniform(0.02, 0.8, n)
    rough[np.isin(kinds, [1, 3])] = 0.0
    m["roughness"] = rough
    m["ior"] = np.where(kinds == 6, 1.33, rng.uniform(1.2, 1.9, n))
    m["intensity"] = 1.0
    m["absorb"] = rng.uniform(0.0, 0.5, (n, 3))
    m["waveAmp"] = 0.05
    m["waveFreq"] = 2.0
    return m


def generate(which, n, seed):
    """Seeded inputs for function `which` (bytes + numpy record array)."""
    rng = np.random.default_rng(seed)
    name, din, _ = ITEMS[which]
    a = np.zeros(n, din)
    if which == 1:
        a["seed"] = rng.integers(0, 2**63, n, dtype=np.uint64) * 2 + rng.integers(0, 2, n, dtype=np.uint64)
        a["seq"] = rng.integers(0, 2**63, n, dtype=np.uint64)
        a["seed"][:4] = [0, 1, 7, (1 << 32) | 5]
        a["seq"][:4] = [0, 1, 7, 1]
    elif which == 2:
        a["m"] = random_materials(rng, n)
        nrm = _unit(rng, n)
        a["n"] = nrm
        a["wo"] = _hemi(rng, nrm, 1.0)
        a["wi"] = _unit(rng, n)
        a["albedo"] = rng.uniform(0.0, 1.0, (n, 3))
        a["eta"] = rng.uniform(0.6, 1.6, n)
    elif which == 3:
        a["m"] = random_materials(rng, n)
        nrm = _unit(rng, n)
        a["n"] = nrm
        a["d"] = _hemi(rng, nrm, -1.0)
        a["albedo"] = rng.uniform(0.0, 1.0, (n, 3))
        a["front"] = rng.integers(0, 2, n)
        a["etaExt"] = np.where(rng.random(n) < 0.7, 1.0, 1.33)
        a["state"] = rng.integers(0, 2**63, n, dtype=np.uint64)
        a["inc"] = rng.integers(0, 2**62, n, dtype=np.uint64) * 2 + 1
    elif which == 4:
        a["kind"] = rng.integers(0, 5, n)
        a["o"] = rng.uniform(-3.0, 3.0, (n, 3))
        tgt = rng.uniform(-1.0, 1.0, (n, 3))
        d = tgt - a["o"]
        a["d"] = d * rng.uniform(0.3, 3.0, (n, 1))
        a["tmin"] = 0.0
        a["tmax"] = np.where(rng.random(n) < 0.8, 1e16, rng.uniform(0.1, 2.0, n))
    elif which == 5:
        a["o"] = rng.uniform(-2.0, 2.0, (n, 3))
        a["p0"] = rng.uniform(-1.0, 1.0, (n, 3))
        a["p1"] = rng.uniform(-1.0, 1.0, (n, 3))
        a["p2"] = rng.uniform(-1.0, 1.0, (n, 3))
        w = rng.dirichlet([1, 1, 1], n) * 1.2 - 0.06
        tgt = w[:, :1] * a["p0"] + w[:, 1:2] * a["p1"] + w[:, 2:3] * a["p2"]
        a["d"] = tgt - a["o"]
        a["tmin"] = 0.0
        a["tmax"] = 1e16
    elif which == 6:
        l = np.zeros(n, LIGHT)
        l["kind"] = rng.choice([0, 1, 2, 3, 4], n)
        l["p"] = rng.uniform(-2.0, 2.0, (n, 3))
        u = _unit(rng, n) * rng.uniform(0.2, 1.5, (n, 1))
        t = _unit(rng, n)
        v = np.cross(t, u)
        v = v / np.linalg.norm(v, axis=1, keepdims=True) * np.linalg.norm(u, axis=1, keepdims=True)
        l["u"], l["v"] = u, v
        nn = np.cross(v, u)
        l["n"] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
        l["L"] = rng.uniform(0.5, 20.0, (n, 3))
        l["radius"] = rng.uniform(0.0, 0.5, n)
        l["area"] = 4.0 * np.linalg.norm(np.cross(u, v), axis=1)
        l["dir"] = _unit(rng, n)
        l["twoSided"] = rng.integers(0, 2, n)
        l["texId"] = -1
        l["flameId"] = -1
        a["l"] = l
        a["x"] = rng.uniform(-4.0, 4.0, (n, 3))
        a["state"] = rng.integers(0, 2**63, n, dtype=np.uint64)
        a["inc"] = rng.integers(0, 2**62, n, dtype=np.uint64) * 2 + 1
    elif which == 7:
        f = np.zeros(n, FLAME)
        f["base"] = rng.uniform(-0.5, 0.5, (n, 3))
        f["height"] = rng.uniform(1.0, 3.0, n)
        f["radius"] = rng.uniform(0.3, 1.0, n)
        f["intensity"] = rng.uniform(5.0, 30.0, n)
        f["sigma"] = rng.uniform(0.5, 8.0, n)
        f["noiseScale"] = rng.uniform(1.0, 5.0, n)
        f["seed"] = rng.integers(0, 1000, n)
        f["steps"] = 32
        a["f"] = f
        o = rng.uniform(-3.0, 3.0, (n, 3))
        tgt = f["base"] + np.stack([rng.uniform(-0.8, 0.8, n), rng.uniform(0.0, 2.5, n),
                                    rng.uniform(-0.8, 0.8, n)], -1)
        d = tgt - o
        a["o"] = o
        a["d"] = d / np.linalg.norm(d, axis=1, keepdims=True)
        a["tEnd"] = rng.uniform(0.5, 10.0, n)
        a["skip"] = np.where(rng.random(n) < 0.2, 0, -1)
        a["state"] = rng.integers(0, 2**63, n, dtype=np.uint64)
        a["inc"] = rng.integers(0, 2**62, n, dtype=np.uint64) * 2 + 1
    elif which == 8:
        a["p"] = rng.uniform(-50.0, 50.0, (n, 3))
        a["seed"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        ns = _unit(rng, n)
        a["ns"] = ns
        a["wo"] = _hemi(rng, ns, 1.0)
        a["amp"] = rng.uniform(0.0, 0.2, n)
        a["freq"] = rng.uniform(0.5, 4.0, n)
    elif which == 9:
        a["u"] = rng.random(n).astype(np.float32)
    return a


def cdf_table(seed, m=300):
    """A CDF with flat runs and an exact 1 at the end, plus probe values
    landing on entries (the tie rule of the binary search)."""
    rng = np.random.default_rng(seed)
    w = rng.random(m) ** 3
    w[rng.random(m) < 0.1] = 0.0
    c = np.concatenate([[0.0], np.cumsum(w, dtype=np.float64)])
    c = (c / c[-1]).astype(np.float32)
    c[-1] = 1.0
    return c


def cdf_payload(us, table):
    return us.tobytes() + np.int32(len(table)).tobytes() + table.astype(np.float32).tobytes()
