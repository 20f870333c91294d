"""ORACLE — test infrastructure only (the checker, never the product).

CPU restatement of the guiding network's forward pass, loss and backward
pass (sundog_b200/csrc/guide.cu, guide_net.h), in numpy. With bf16=True it
rounds to BF16 at exactly the points the CUDA kernels do (weights, input
features, each hidden activation after ReLU, the output gradient and each
hidden gradient after the ReLU mask) and accumulates in float64, so the GPU's
FP32-accumulated results differ from it only by accumulation order and the
rare BF16 rounding flip that follows. With bf16=False everything is float64:
the tests check that variant's analytic gradient against finite differences,
which pins the loss-gradient formulas themselves.

The reference has no learned guiding; there is nothing of it to pin against.
"""

import numpy as np

N_IN, N_HID, N_OUT, N_LOBE_OUT = 48, 64, 48, 40
FREQS = 5
LOBES = 8
KAPPA_MIN, KAPPA_MAX = 0.05, 500.0
WEIGHT_CLAMP = 100.0

OFF_W0 = 0
OFF_W1 = OFF_W0 + N_HID * N_IN
OFF_W2 = OFF_W1 + N_HID * N_HID
OFF_W3 = OFF_W2 + N_HID * N_HID
N_WEIGHTS = OFF_W3 + N_OUT * N_HID
OFF_B0 = N_WEIGHTS
OFF_B1 = OFF_B0 + N_HID
OFF_B2 = OFF_B1 + N_HID
OFF_B3 = OFF_B2 + N_HID
N_PARAMS = OFF_B3 + N_OUT


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, bf=True):
    p = np.asarray(params, np.float64)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    W0 = r(p[OFF_W0:OFF_W1].reshape(N_HID, N_IN))
    W1 = r(p[OFF_W1:OFF_W2].reshape(N_HID, N_HID))
    W2 = r(p[OFF_W2:OFF_W3].reshape(N_HID, N_HID))
    W3 = r(p[OFF_W3:N_WEIGHTS].reshape(N_OUT, N_HID))
    b = [np.asarray(p[OFF_B0:OFF_B1], np.float64), np.asarray(p[OFF_B1:OFF_B2], np.float64),
         np.asarray(p[OFF_B2:OFF_B3], np.float64), np.asarray(p[OFF_B3:N_PARAMS], np.float64)]
    return [W0, W1, W2, W3], b


def features(pos, nrm, bf=True):
    """48 inputs per row: sin/cos(2^j pi p_i) at columns 10 i + 2 j (+1),
    zeros at 30-31, the normal at 32-34, zeros after."""
    pos = np.asarray(pos, np.float64)
    nrm = np.asarray(nrm, np.float64)
    f = np.zeros((pos.shape[0], N_IN))
    for i in range(3):
        for j in range(FREQS):
            v = pos[:, i] * (1 << j)
            f[:, 10 * i + 2 * j] = np.sin(np.pi * v)
            f[:, 10 * i + 2 * j + 1] = np.cos(np.pi * v)
    f[:, 32:35] = nrm
    return bf16(f) if bf else f


def forward(params, pos, nrm, bf=True):
    W, b = unpack(params, bf)
    r = bf16 if bf else (lambda a: a)
    x = features(pos, nrm, bf)
    h0 = r(np.maximum(x @ W[0].T + b[0], 0.0))
    h1 = r(np.maximum(h0 @ W[1].T + b[1], 0.0))
    h2 = r(np.maximum(h1 @ W[2].T + b[2], 0.0))
    out = h2 @ W[3].T + b[3]
    return out, (x, h0, h1, h2)


def decode(o):
    """Per-row lobes from the 40 used outputs: mu (N,8,3), kappa, log w,
    |r| and d kappa / d s (0 where kappa is clamped)."""
    o = np.asarray(o, np.float64)[:, :N_LOBE_OUT].reshape(-1, LOBES, 5)
    r = o[:, :, :3]
    rn = np.maximum(np.linalg.norm(r, axis=-1), 1e-4)
    mu = r / rn[..., None]
    s = o[:, :, 3]
    sp = np.where(s > 15.0, s, np.log1p(np.exp(np.minimum(s, 15.0))))
    kappa = sp + KAPPA_MIN
    dk = 1.0 / (1.0 + np.exp(-s))
    clamped = kappa > KAPPA_MAX
    kappa = np.where(clamped, KAPPA_MAX, kappa)
    dk = np.where(clamped, 0.0, dk)
    z = o[:, :, 4]
    zmax = z.max(axis=1, keepdims=True)
    logw = z - (zmax + np.log(np.exp(z - zmax).sum(axis=1, keepdims=True)))
    return mu, kappa, logw, rn, dk


def vmf_log_norm(kappa):
    return np.log(kappa) - np.log(2.0 * np.pi) - np.log1p(-np.exp(-2.0 * kappa))


def mixture_log_density(o, w):
    mu, kappa, logw, _, _ = decode(o)
    cosm = np.einsum("nkc,nc->nk", mu, w)
    lq = logw + vmf_log_norm(kappa) + kappa * (cosm - 1.0)
    m = lq.max(axis=1, keepdims=True)
    return (m + np.log(np.exp(lq - m).sum(axis=1, keepdims=True)))[:, 0]


def head_loss_grad(o, w, c):
    """Loss sum_i -c_i log q_i and d loss / d outputs (N, 48)."""
    mu, kappa, logw, rn, dk = decode(o)
    w = np.asarray(w, np.float64)
    cosm = np.einsum("nkc,nc->nk", mu, w)
    lq = logw + vmf_log_norm(kappa) + kappa * (cosm - 1.0)
    m = lq.max(axis=1, keepdims=True)
    logq = m + np.log(np.exp(lq - m).sum(axis=1, keepdims=True))
    gam = np.exp(lq - logq)
    wk = np.exp(logw)
    c = np.asarray(c, np.float64)[:, None]
    d = np.zeros((o.shape[0], LOBES, 5))
    d[:, :, 4] = -c * (gam - wk)
    dlk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (cosm - 1.0)
    d[:, :, 3] = -c * gam * dlk * dk
    d[:, :, :3] = (w[:, None, :] - cosm[..., None] * mu) * (-c * gam * kappa / rn)[..., None]
    out = np.zeros((o.shape[0], N_OUT))
    out[:, :N_LOBE_OUT] = d.reshape(-1, N_LOBE_OUT)
    return float(-(c[:, 0] * logq[:, 0]).sum()), out


def record_weights(F):
    """c_i = min(F_i / mean(F), clamp) / batch."""
    F = np.asarray(F, np.float64)
    return np.minimum(F / F.mean(), WEIGHT_CLAMP) / len(F)


def loss_and_grads(params, records, box, bf=True):
    """Loss and parameter gradient (N_PARAMS,) over records (N x 12:
    x, F, n, 0, wi, 0); box = (lo.xyz, 1/extent.xyz)."""
    rec = np.asarray(records, np.float64).reshape(-1, 12)
    lo, inv = np.asarray(box[:3], np.float64), np.asarray(box[3:6], np.float64)
    pos = np.clip((rec[:, 0:3] - lo) * inv, 0.0, 1.0)
    nrm, wi, F = rec[:, 4:7], rec[:, 8:11], rec[:, 3]
    W, b = unpack(params, bf)
    r = bf16 if bf else (lambda a: a)
    out, (x, h0, h1, h2) = forward(params, pos, nrm, bf)
    loss, dO = head_loss_grad(out, wi, record_weights(F))
    dO = r(dO)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:N_WEIGHTS] = (dO.T @ h2).ravel()
    g[OFF_B3:N_PARAMS] = dO.sum(0)
    dZ2 = r((dO @ W[3]) * (h2 > 0))
    g[OFF_W2:OFF_W3] = (dZ2.T @ h1).ravel()
    g[OFF_B2:OFF_B3] = dZ2.sum(0)
    dZ1 = r((dZ2 @ W[2]) * (h1 > 0))
    g[OFF_W1:OFF_W2] = (dZ1.T @ h0).ravel()
    g[OFF_B1:OFF_B2] = dZ1.sum(0)
    dZ0 = r((dZ1 @ W[1]) * (h0 > 0))
    g[OFF_W0:OFF_W1] = (dZ0.T @ x).ravel()
    g[OFF_B0:OFF_B1] = dZ0.sum(0)
    return loss, g


def init_params(seed):
    """A random parameter vector (not the library's initialisation): He
    normal weights, small random biases, output biases as the library sets
    them (lobes toward the cube corners, kappa 2, equal weights)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS)
    p[OFF_W0:OFF_W1] = rng.standard_normal(OFF_W1 - OFF_W0) * np.sqrt(2.0 / 35.0)
    p[OFF_W1:OFF_W3] = rng.standard_normal(OFF_W3 - OFF_W1) * np.sqrt(2.0 / N_HID)
    p[OFF_W3:N_WEIGHTS] = rng.standard_normal(N_WEIGHTS - OFF_W3) * 0.05
    p[OFF_B0:OFF_B3] = rng.standard_normal(OFF_B3 - OFF_B0) * 0.05
    d = 1.0 / np.sqrt(3.0)
    for k in range(LOBES):
        p[OFF_B3 + 5 * k:OFF_B3 + 5 * k + 3] = [d if k & 1 else -d, d if k & 2 else -d,
                                                 d if k & 4 else -d]
        p[OFF_B3 + 5 * k + 3] = np.log(np.exp(2.0 - KAPPA_MIN) - 1.0)
    return p.astype(np.float32)


def random_records(n, seed, lo=(-2.0, -1.0, -3.0), hi=(3.0, 2.0, 1.0)):
    """n synthetic training records inside the box lo..hi."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    rec = np.zeros((n, 12), np.float32)
    rec[:, 0:3] = lo + (hi - lo) * rng.random((n, 3))
    rec[:, 3] = rng.exponential(1.0, n) * (rng.random(n) < 0.8)  + 1e-3
    nv = rng.standard_normal((n, 3))
    rec[:, 4:7] = nv / np.linalg.norm(nv, axis=1, keepdims=True)
    wv = rng.standard_normal((n, 3)) + 0.8 * rec[:, 4:7]
    rec[:, 8:11] = wv / np.linalg.norm(wv, axis=1, keepdims=True)
    box = np.concatenate([lo, 1.0 / (hi - lo)]).astype(np.float32)
    return rec, box
