"""Learned path guiding on the GPU.

  * the network's forward outputs and its loss gradient (BF16 operands, FP32
    accumulation on the tensor cores) against the CPU oracle's restatement
    (oracle/guide_mlp.py), which rounds to BF16 at the same points; the
    remaining difference is accumulation order plus the BF16 rounding flips
    it causes, bounded per quantity below;
  * guided rendering is unbiased: its image agrees with the plain kernel's
    within Monte Carlo noise;
  * what the trained network gains (cross-entropy of its mixture against
    the sampling target, and image error at equal spp) on the
    flame/water/glass scene at reduced resolution.
"""

import ctypes
import numpy as np
import pytest

from oracle import guide_mlp as gm
from sundog_b200 import abi
from sundog_b200 import scene as sc
from sundog_b200 import workloads

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_init_params(lib):
    p = np.zeros(abi.GUIDE_PARAMS, np.float32)
    abi.check(lib.sundog_guide_init_params(1, p.ctypes.data), "init", lib)
    assert np.isfinite(p).all()
    b3 = p[gm.OFF_B3:].reshape(-1)[:40].reshape(8, 5)
    assert np.allclose(np.abs(b3[:, :3]), 1 / np.sqrt(3), atol=1e-6)
    assert np.allclose(b3[:, 4], 0.0)
    q = np.zeros_like(p)
    abi.check(lib.sundog_guide_init_params(1, q.ctypes.data), "init", lib)
    assert np.array_equal(p, q)


def test_forward_parity(lib):
    params = gm.init_params(11)
    rng = np.random.default_rng(12)
    n = 1000
    pos = rng.random((n, 3))
    nv = rng.standard_normal((n, 3))
    nrm = nv / np.linalg.norm(nv, axis=1, keepdims=True)
    q = np.concatenate([pos, nrm], 1).astype(np.float32)
    out = np.zeros((n, 40), np.float32)
    abi.check(lib.sundog_guide_outputs(params.ctypes.data, q.ctypes.data, n, out.ctypes.data),
              "outputs", lib)
    ref, _ = gm.forward(params, q[:, :3], q[:, 3:], bf=True)
    ref = ref[:, :40]
    e = relerr(out, ref)
    print("forward: relative error %.2e" % e)
    # FP32 vs float64 accumulation of BF16 products; a hidden activation that
    # lands on the other side of a BF16 rounding boundary moves by 2^-8.
    assert e <= 5e-3
    lq_g = gm.mixture_log_density(out.astype(np.float64), nrm)
    lq_o = gm.mixture_log_density(ref, nrm)
    assert np.max(np.abs(lq_g - lq_o)) <= 2e-2


@pytest.mark.parametrize("n", [128, 1000, 5000])
def test_gradient_parity(lib, n):
    params = gm.init_params(21 + n)
    rec, box = gm.random_records(n, 22 + n)
    grads = np.zeros(abi.GUIDE_PARAMS, np.float32)
    loss = ctypes.c_float(0.0)
    abi.check(lib.sundog_guide_gradients(params.ctypes.data, rec.ctypes.data, n, box.ctypes.data,
                                         grads.ctypes.data, ctypes.byref(loss)), "gradients", lib)
    l_ref, g_ref = gm.loss_and_grads(params, rec, box, bf=True)
    print("n=%d loss gpu %.6f oracle %.6f" % (n, loss.value, l_ref))
    assert abs(loss.value - l_ref) <= 2e-3 * abs(l_ref)
    layers = [("W0", gm.OFF_W0, gm.OFF_W1), ("W1", gm.OFF_W1, gm.OFF_W2),
              ("W2", gm.OFF_W2, gm.OFF_W3), ("W3", gm.OFF_W3, gm.N_WEIGHTS),
              ("b0", gm.OFF_B0, gm.OFF_B1), ("b1", gm.OFF_B1, gm.OFF_B2),
              ("b2", gm.OFF_B2, gm.OFF_B3), ("b3", gm.OFF_B3, gm.N_PARAMS)]
    for name, lo, hi in layers:
        g, o = grads[lo:hi].astype(np.float64), g_ref[lo:hi]
        e = relerr(g, o)
        cos = float(g @ o / max(np.linalg.norm(g) * np.linalg.norm(o), 1e-30))
        print("  %s: relative error %.2e  cosine %.6f" % (name, e, cos))
        # BF16 gradient operands (2^-8 relative) summed over up to 5000
        # records in a different order.
        assert e <= 2e-2, name
        assert cos >= 0.9995, name


def test_guided_render_unbiased(lib):
    s = workloads.cornell(width=64, height=64, spp=512)
    with sc.Session(s) as plain:
        plain.render()
        fp = plain.read()[..., :3].astype(np.float64)
    with sc.Session(s) as guided:
        guided.set_guiding(True, train_spp=32, pass_spp=8, steps_per_pass=32, batch=8192)
        guided.render()
        st = guided.guiding_stats()
        fg = guided.read()[..., :3].astype(np.float64)
    assert st.passes == 4 and st.train_steps == 128 and st.records > 0
    assert np.isfinite(fg).all()
    mp, mg = fp.mean(axis=(0, 1)), fg.mean(axis=(0, 1))
    print("plain mean %s guided mean %s" % (mp, mg))
    assert np.all(np.abs(mg - mp) <= 0.02 * mp)
    # 8x8-pixel blocks: agreement within the blocks' own noise.
    bp = fp.reshape(8, 8, 8, 8, 3).mean(axis=(1, 3))
    bg = fg.reshape(8, 8, 8, 8, 3).mean(axis=(1, 3))
    rel = np.abs(bg - bp) / np.maximum(bp, 1e-3)
    assert np.median(rel) <= 0.03 and np.quantile(rel, 0.95) <= 0.15


def test_record_pass_engines_agree(lib, asset_dir):
    """A training pass records the same samples on both engines: the first
    pass (no guide yet) traces the plain paths, and each guided vertex
    becomes one record when its path ends, whether the path's trail lives in
    the megakernel thread or in its wavefront slot. Record order follows
    atomics, so the record sets are compared sorted."""
    s = workloads.volumes(asset_dir, width=96, height=54, spp=4)
    recs = []
    for engine in (0, 1):
        with sc.Session(s, base_dir=asset_dir, engine=engine) as ses:
            ses.set_guiding(True, train_spp=4, pass_spp=4, steps_per_pass=1)
            ses.render()
            assert ses.guiding_stats().passes == 1
            recs.append(ses.guide_records(1 << 20).astype(np.float64))
    a, b = recs
    print("records: wavefront %d, megakernel %d" % (len(a), len(b)))
    assert len(a) == len(b) > 1000
    for col in (3, 0, 1, 2, 4, 5, 6, 8, 9, 10):  # F, x, n, wi
        sa, sb = np.sort(a[:, col]), np.sort(b[:, col])
        scale = max(np.abs(sa).max(), 1e-6)
        assert np.quantile(np.abs(sa - sb), 0.99) <= 1e-4 * scale, col
        assert abs(sa.sum() - sb.sum()) <= 1e-4 * np.abs(sa).sum() + 1e-6, col


def _relmse_map(img, ref):
    img = img[..., :3].astype(np.float64)
    ref = ref[..., :3].astype(np.float64)
    return ((img - ref) ** 2 / (ref ** 2 + 1e-2)).mean(-1)


def _relmse(img, ref):
    img = img[..., :3].astype(np.float64)
    ref = ref[..., :3].astype(np.float64)
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def test_trained_network_gain(lib, asset_dir):
    """What the trained network gains over the method without it, on the
    flame / water / glass scene (640x360):
      * as a sampling distribution: on the last training pass's records its
        cross-entropy against the target (incident radiance x |cos|) is far
        below that of the BSDF-only (cosine) sampler and of its own
        untrained start;
      * in the image: at equal spp, relative MSE against a 1024-spp plain
        render is lower with guiding than without over the image's bulk
        (pixels below the 99th percentile of either render's error; the top
        pixels hold glints of the flame's point lights on a glossy panel,
        drawn before any guided vertex and shared by both renders), and the
        guided image has the plain image's mean (same expectation).
    Equal-time figures are reported by bench.py --guiding."""
    w, h = 640, 360
    with sc.Session(workloads.volumes(asset_dir, width=w, height=h, spp=1024),
                    base_dir=asset_dir) as r:
        r.render()
        ref = r.read()
    s = workloads.volumes(asset_dir, width=w, height=h, spp=64)
    with sc.Session(s, base_dir=asset_dir) as g:
        g.set_guiding(True)
        res_g = g.render()
        img_g = g.read()
        st = g.guiding_stats()
        params = g.guide_params()
        rec = g.guide_records(1 << 17).astype(np.float64)
    with sc.Session(s, base_dir=asset_dir) as p:
        res_p = p.render()
        img_p = p.read()
    assert len(rec) > 10000 and st.passes == 4
    lo, hi = np.array(st.box_lo, np.float64), np.array(st.box_hi, np.float64)
    pos = np.clip((rec[:, 0:3] - lo) / (hi - lo), 0.0, 1.0)
    nrm, wi, F = rec[:, 4:7], rec[:, 8:11], rec[:, 3]
    c = F / F.sum()
    init = np.zeros(abi.GUIDE_PARAMS, np.float32)
    abi.check(lib.sundog_guide_init_params(1, init.ctypes.data), "init", lib)
    ce = lambda prm: -float(np.sum(c * gm.mixture_log_density(
        gm.forward(prm, pos, nrm, bf=True)[0], wi)))
    cos = np.maximum(np.sum(wi * nrm, 1), 1e-12)
    ce_cos = -float(np.sum(c * np.log(cos / np.pi)))
    ce_trained, ce_init = ce(params), ce(init)
    e_g, e_p = _relmse(img_g, ref), _relmse(img_p, ref)
    mg_, mp_ = _relmse_map(img_g, ref), _relmse_map(img_p, ref)
    both = np.maximum(mg_, mp_)
    keep = both <= np.quantile(both, 0.99)
    b_g, b_p = float(mg_[keep].mean()), float(mp_[keep].mean())
    print("cross-entropy (nats): trained %.3f  untrained %.3f  cosine %.3f" %
          (ce_trained, ce_init, ce_cos))
    print("64 spp: relMSE guided %.4g (%.1f ms incl. %.1f ms training)  plain %.4g (%.1f ms); "
          "bulk guided %.4g plain %.4g" %
          (e_g, res_g.render_ms, st.train_ms, e_p, res_p.render_ms, b_g, b_p))
    assert ce_trained < ce_cos - 0.5 and ce_trained < ce_init - 1.0
    assert b_g < 0.8 * b_p
    mg, mp = img_g[..., :3].mean(axis=(0, 1)), img_p[..., :3].mean(axis=(0, 1))
    assert np.all(np.abs(mg - mp) <= 0.01 * mp)
