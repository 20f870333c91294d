"""The allocation-free tile render (sundog_session_render_tile_noalloc).

It exists for callers that cannot allocate device memory while they render
(a worker whose device memory belongs to another allocator or is held to a
fixed budget); its scratch is a static device array inside the library.
Here the caller's film is a torch tensor (memory the caller already owns).
Checked against the existing entry point (a full render of the same session
read back with sundog_session_read) on consecutive calls that reuse the
shared scratch: a sub-tile, the whole image, and a two-call sample split,
each within the per-pixel tolerance of the render parity tests (1e-3
relative; the paths are the same paths, so they match exactly in practice).
"""

import ctypes

import numpy as np
import pytest

from sundog_b200 import scene as sc
from sundog_b200 import workloads

pytestmark = pytest.mark.gpu


def tile(lib, ses, x0, y0, w, h, s0, n, film=None):
    import torch
    if film is None:
        film = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    rays = ctypes.c_uint64(0)
    torch.cuda.synchronize()
    rc = lib.sundog_session_render_tile_noalloc(ses.handle, x0, y0, w, h, s0, n, film.data_ptr(),
                                                ctypes.byref(rays), None)
    assert rc == 0, lib.sundog_last_error()
    return film, rays.value


def close(got, ref):
    got = got[..., :3].astype(np.float64)
    ref = ref[..., :3].astype(np.float64)
    scale = np.maximum(np.maximum(np.abs(got), np.abs(ref)), 1e-2)
    ok = np.all(np.abs(got - ref) <= 1e-3 * scale, axis=-1)
    return ok.mean()


def test_tile_noalloc_matches_full_render(lib):
    torch = pytest.importorskip("torch")
    s = workloads.cornell(width=64, height=48, spp=16)
    with sc.Session(s) as ses:
        full_res = ses.render()
        full = ses.read()
        # first call: a sub-rectangle
        f1, r1 = tile(lib, ses, 8, 4, 40, 24, 0, 16)
        assert close(f1.cpu().numpy(), full[4:28, 8:48]) == 1.0
        assert r1 > 0
        # second call in a row, reusing the scratch: the whole image; the
        # ray count then equals the full render's
        f2, r2 = tile(lib, ses, 0, 0, 64, 48, 0, 16)
        assert close(f2.cpu().numpy(), full) == 1.0
        assert r2 == full_res.rays_traced
        # samples split over two calls fold into the same film
        f3, _ = tile(lib, ses, 16, 16, 32, 16, 0, 9)
        f3, _ = tile(lib, ses, 16, 16, 32, 16, 9, 7, film=f3)
        assert close(f3.cpu().numpy(), full[16:32, 16:48]) == 1.0


def test_tile_noalloc_rejects_oversized_and_outside(lib):
    torch = pytest.importorskip("torch")
    s = workloads.cornell(width=64, height=48, spp=16)
    with sc.Session(s) as ses:
        film = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
        rc = lib.sundog_session_render_tile_noalloc(ses.handle, 0, 0, 64, 48, 0, 400,
                                                    film.data_ptr(), None, None)
        assert rc != 0 and b"exceeds" in lib.sundog_last_error()
        rc = lib.sundog_session_render_tile_noalloc(ses.handle, 40, 0, 32, 16, 0, 4,
                                                    film.data_ptr(), None, None)
        assert rc != 0 and b"outside" in lib.sundog_last_error()


def test_tile_noalloc_follows_session_sample_offset(lib):
    """A session created with a sample offset draws samples offset..offset+spp;
    the tile call counts its sample_begin from that offset too."""
    torch = pytest.importorskip("torch")
    s = workloads.cornell(width=48, height=32, spp=8)
    with sc.Session(s, sample_offset=5) as ses:
        ses.render()
        full = ses.read()
        f, _ = tile(lib, ses, 0, 0, 48, 32, 0, 8)
        assert close(f.cpu().numpy(), full) == 1.0
    with sc.Session(s) as plain:
        plain.render()
        assert not np.array_equal(plain.read(), full)


def test_tile_noalloc_rejects_guided_session(lib):
    torch = pytest.importorskip("torch")
    s = workloads.cornell(width=32, height=32, spp=4)
    with sc.Session(s) as ses:
        ses.set_guiding(True)
        film = torch.zeros((32, 32, 4), dtype=torch.float32, device="cuda")
        rc = lib.sundog_session_render_tile_noalloc(ses.handle, 0, 0, 32, 32, 0, 4,
                                                    film.data_ptr(), None, None)
        assert rc != 0 and b"guiding" in lib.sundog_last_error()
