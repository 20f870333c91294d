"""ORACLE — test infrastructure only (the checker, never the product).

numpy restatement of sundog's sampling-table builds in FP64:

  env_tables     the equirect map's marginal and conditional CDFs over
                 luminance * sin(theta) (src/env_light.cpp:27-56);
  mesh_light_cdf the world-space triangle-area CDF of an emissive mesh
                 instance (src/capi_render.cpp:126-155).

Each returns the tables as the reference stores them (FP32 values of the
sequential FP64 prefix sums, normalised in FP64; numpy's cumsum adds in
sequence, so these are the reference's tables bit for bit given the same
inputs) and the unrounded FP64 values of the same quantities (prefix / total
before any float rounding), against which a table's error is measured.
read_rgbe decodes the flat Radiance files the workloads write.
"""

import ctypes
import ctypes.util

import numpy as np

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]


def _sinf(x):
    return _libm.sinf(x)


def read_rgbe(path):
    """Flat (non-RLE) Radiance RGBE file -> float32 (H, W, 3), row 0 = top."""
    with open(path, "rb") as f:
        data = f.read()
    head, _, rest = data.partition(b"\n\n")
    line, _, pix = rest.partition(b"\n")
    parts = line.split()
    h, w = int(parts[1]), int(parts[3])
    a = np.frombuffer(pix[:h * w * 4], np.uint8).reshape(h, w, 4).astype(np.int32)
    e = a[..., 3]
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    return (a[..., :3] * scale[..., None]).astype(np.float32)


def _normalised(prefix32, total):
    """Reference normalisation: float prefix / FP64 total, as float; last = 1."""
    out = (prefix32.astype(np.float64) / total).astype(np.float32)
    out[0] = 0.0
    out[-1] = 1.0
    return out


def env_tables(rgb):
    """rgb: float32 (H, W, 3). Returns (marg, cond, marg64, cond64): marg
    (H + 1) and cond (H, W + 1) as the reference stores them, and the FP64
    prefix / total of each without float rounding."""
    rgb = np.asarray(rgb, np.float32)
    h, w, _ = rgb.shape
    f = np.float32
    lum = (f(0.2126) * rgb[..., 0] + f(0.7152) * rgb[..., 1]) + f(0.0722) * rgb[..., 2]
    lum = np.where(lum > 0, lum, f(0.0)).astype(np.float32)
    rows = np.arange(h, dtype=np.float32)
    # sinf(pi * (row + 0.5) / h) with FP32 arguments, through the C library's
    # sinf as the reference calls it (it is not correctly rounded for every
    # argument, and the tables follow it).
    arg = (f(np.pi) * (rows + f(0.5))) / f(h)
    sin_t = np.array([_sinf(float(a)) for a in arg], np.float32)
    vals = lum.astype(np.float64) * sin_t.astype(np.float64)[:, None]
    cond = np.zeros((h, w + 1), np.float32)
    cond64 = np.zeros((h, w + 1), np.float64)
    sums = np.zeros(h, np.float64)
    for r in range(h):
        pre = np.cumsum(vals[r])
        sums[r] = pre[-1]
        if sums[r] > 0:
            row = np.concatenate([[0.0], pre.astype(np.float32).astype(np.float64)])
            cond[r] = _normalised(row.astype(np.float32), sums[r])
            cond64[r, 1:] = pre / sums[r]
        else:
            cond[r] = (np.arange(w + 1, dtype=np.float32) / f(w)).astype(np.float32)
            cond64[r] = np.arange(w + 1) / w
        cond[r, w] = 1.0
        cond64[r, w] = 1.0
    tot = np.cumsum(sums)
    if tot[-1] > 0:
        marg = _normalised(np.concatenate([[0.0], tot]).astype(np.float32), tot[-1])
        marg64 = np.concatenate([[0.0], tot / tot[-1]])
    else:
        marg = (np.arange(h + 1, dtype=np.float32) / f(h)).astype(np.float32)
        marg64 = np.arange(h + 1) / h
    marg[h] = 1.0
    return marg, cond, marg64, cond64


def read_obj_triangles(path):
    """Vertex positions (float32) and triangle indices of a plain OBJ (the
    workloads' meshes: 'v' and 'f' records, polygons fanned)."""
    pos, tris = [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "v":
                pos.append([float(x) for x in p[1:4]])
            elif p[0] == "f":
                idx = [int(x.split("/")[0]) - 1 for x in p[1:]]
                for k in range(1, len(idx) - 1):
                    tris.append([idx[0], idx[k], idx[k + 1]])
    return np.array(pos, np.float32), np.array(tris, np.int64)


def mesh_light_cdf(pos, tris, xform12):
    """World vertices = xform (3x4, row-major, FP32, the reference's
    m0 x + m1 y + m2 z + m3 order), areas 0.5 |e1 x e2| in FP32 widened to
    FP64, sequential FP64 prefix. Returns (cdf, cdf64, total)."""
    m = np.asarray(xform12, np.float32)
    p = np.asarray(pos, np.float32)
    wp = np.stack([((m[4 * r] * p[:, 0] + m[4 * r + 1] * p[:, 1]) + m[4 * r + 2] * p[:, 2])
                   + m[4 * r + 3] for r in range(3)], -1).astype(np.float32)
    a, b, c = wp[tris[:, 0]], wp[tris[:, 1]], wp[tris[:, 2]]
    u, v = b - a, c - a
    cx = u[:, 1] * v[:, 2] - u[:, 2] * v[:, 1]
    cy = u[:, 2] * v[:, 0] - u[:, 0] * v[:, 2]
    cz = u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]
    ln = np.sqrt((cx * cx + cy * cy) + cz * cz).astype(np.float32)
    area = 0.5 * ln.astype(np.float64)
    pre = np.cumsum(area)
    total = pre[-1]
    cdf = _normalised(np.concatenate([[0.0], pre]).astype(np.float32), total)
    cdf64 = np.concatenate([[0.0], pre / total])
    cdf64[-1] = 1.0
    return cdf, cdf64, total
