"""The film denoiser (denoise.cu), the replacement of the reference's
optional OptiX denoiser pass (src/denoise.cpp:18-53, src/capi_render.cpp:
247-256), judged the way the reference judges its own (docs/BENCHMARKS.md
tier B: error of a low-spp film against a high-spp render of the same scene):
relative MSE per pixel, (x - ref)^2 / (ref^2 + 0.01), RGB mean.

Bounds: the denoised 16-spp film has at most 0.6 of the raw film's error
(measured on these scenes when the filter was tuned: 13.9x lower on the
Cornell box, 2.1x on the image-texture scene, whose raw error is already
small); its
mean brightness stays within 3% of the raw film's (the filter redistributes
radiance, it does not add or remove it); sundog_render_ex with denoise on
returns exactly what sundog_session_denoise returns for the same film."""

import ctypes

import numpy as np
import pytest

from sundog_b200 import abi, workloads
from sundog_b200 import scene as sc

pytestmark = pytest.mark.gpu


def relmse(x, ref):
    x = x[..., :3].astype(np.float64)
    ref = ref[..., :3].astype(np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


@pytest.mark.parametrize("name", ["cornell", "textured"])
def test_denoiser_lowers_error(lib, asset_dir, name):
    make = {"cornell": lambda spp: workloads.cornell(width=128, height=128, spp=spp),
            "textured": lambda spp: workloads.textured(asset_dir, spp=spp)}[name]
    with sc.Session(make(2048), base_dir=asset_dir, seed=99) as r:
        r.render()
        ref = r.read()
    with sc.Session(make(16), base_dir=asset_dir, aov=True) as ses:
        ses.render()
        raw, _, _ = ses.read()
        den = ses.denoise()
    e_raw, e_den = relmse(raw, ref), relmse(den, ref)
    m_raw, m_den = raw[..., :3].mean(), den[..., :3].mean()
    print("%s: relMSE raw %.4e denoised %.4e (%.2fx lower); mean %.5f -> %.5f"
          % (name, e_raw, e_den, e_raw / e_den, m_raw, m_den))
    assert np.isfinite(den).all()
    assert e_den <= 0.6 * e_raw
    assert abs(m_den - m_raw) <= 0.03 * m_raw


def test_render_option_returns_denoised_film(lib):
    s = workloads.cornell(width=64, height=64, spp=8)
    h = s.build(".", lib)
    try:
        film = np.zeros((64, 64, 4), np.float32)
        o = abi.options(quiet=True, denoise=1)
        ext = abi.RenderExt(film.ctypes.data, None, None, 0, 1, 0, 0, 0, 0)
        res = abi.RenderResult()
        abi.check(lib.sundog_render_ex(h, ctypes.byref(o), ctypes.byref(ext), ctypes.byref(res)),
                  "render", lib)
    finally:
        lib.sundog_scene_destroy(h)
    with sc.Session(s, aov=True) as ses:
        ses.render()
        den = ses.denoise()
    assert film.tobytes() == den.tobytes()
