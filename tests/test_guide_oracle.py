"""CPU checks of the guiding network's oracle (oracle/guide_mlp.py).

The float64 variant's analytic gradient must equal central finite
differences of its own loss, which pins the loss-gradient formulas (softmax
weights, softplus concentrations, normalised directions, vMF normaliser)
that the CUDA head restates. The BF16 variant must stay close to the
float64 one (rounding only).
"""

import numpy as np

from oracle import guide_mlp as gm


def test_gradient_matches_finite_differences():
    params = gm.init_params(3).astype(np.float64)
    rec, box = gm.random_records(64, 5)
    loss, g = gm.loss_and_grads(params, rec, box, bf=False)
    assert np.isfinite(loss) and np.isfinite(g).all()
    rng = np.random.default_rng(7)
    picks = []
    for lo, hi in [(gm.OFF_W0, gm.OFF_W1), (gm.OFF_W1, gm.OFF_W2), (gm.OFF_W2, gm.OFF_W3),
                   (gm.OFF_W3, gm.N_WEIGHTS), (gm.OFF_B0, gm.OFF_B1), (gm.OFF_B3, gm.N_PARAMS)]:
        picks += list(rng.integers(lo, hi, 6))
    # Output biases of every lobe field (r, s, z) explicitly.
    picks += [gm.OFF_B3 + 5 * 2 + j for j in range(5)]
    eps = 1e-6
    for i in picks:
        p1 = params.copy()
        p1[i] += eps
        p0 = params.copy()
        p0[i] -= eps
        fd = (gm.loss_and_grads(p1, rec, box, bf=False)[0] -
              gm.loss_and_grads(p0, rec, box, bf=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 65504.0, 1e-30], np.float32)
    r = gm.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0           # tie -> even mantissa
    assert r[2] == 1.0078125     # above the tie -> up
    assert abs(r[3] + 3.140625) < 1e-12
    bits = r.astype(np.float32).view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)


def test_bf16_variant_close_to_fp64():
    params = gm.init_params(4)
    rec, box = gm.random_records(256, 6)
    l64, g64 = gm.loss_and_grads(params, rec, box, bf=False)
    l16, g16 = gm.loss_and_grads(params, rec, box, bf=True)
    assert abs(l16 - l64) <= 2e-2 * abs(l64)
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)


def test_mixture_is_normalised():
    params = gm.init_params(8)
    pos = np.random.default_rng(1).random((4, 3))
    nrm = np.tile([0.0, 1.0, 0.0], (4, 1))
    out, _ = gm.forward(params, pos, nrm, bf=False)
    # Monte Carlo over uniform directions: E[q / (1 / 4 pi)] = 1.
    rng = np.random.default_rng(2)
    w = rng.standard_normal((200000, 3))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    for r in range(4):
        lq = gm.mixture_log_density(np.repeat(out[r:r + 1], len(w), 0), w)
        est = np.mean(np.exp(lq)) * 4 * np.pi
        assert abs(est - 1.0) < 0.02, est
