"""Float64 reference of the path-guiding model.  TEST INFRASTRUCTURE ONLY (the checker of the CUDA
guiding kernels); the reference renderer has no guiding, so this restates the method the library
implements:

* input encoding (96 features): position normalised to the scene box, 12 "one-blob" bins per axis with a
  triangle kernel (value max(0, 1 - |12 x - (i + 1/2)|)); the shading normal and the outgoing direction as
  (theta / pi, (phi + pi) / 2pi), 12 bins each; feature 84 = 1; features 85..95 = 0.
* MLP 96 -> 64 -> 64 -> 64 -> 64 -> 48, ReLU on the four hidden layers, weights W[out][in] and biases.
* output: 8 von Mises-Fisher lobes, 5 raw values each (logit, mean xyz, concentration): weights =
  softmax(logits), mean = normalised xyz, kappa = min(softplus(raw) + 0.05, 2000).
  vMF(w) = kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu . w - 1)).
* loss over a batch of radiance samples (w_j = target / sampling pdf, wi_j): the Monte-Carlo KL
  divergence  L = -(1/B) sum_j (w_j / mean(w)) log q(wi_j)  and its gradient.
* Adam (beta1 0.9, beta2 0.99, eps 1e-8).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, LOBES = 96, 64, 48, 8
LAYERS = [(IN, HID), (HID, HID), (HID, HID), (HID, HID), (HID, OUT)]
KAPPA_MIN, KAPPA_MAX = 0.05, 2000.0
BETA1, BETA2, EPS = 0.9, 0.99, 1e-8


def param_count() -> int:
    return sum(o * i + o for i, o in LAYERS)


def unpack(params):
    """Flat fp32/64 vector -> [(W[out][in], b[out])] in layer order (W then b per layer)."""
    out, k = [], 0
    for i, o in LAYERS:
        W = params[k:k + o * i].reshape(o, i)
        k += o * i
        b = params[k:k + o]
        k += o
        out.append((W, b))
    return out


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases (the layout of pb2_guide_get_params)."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, o in LAYERS:
        lim = np.sqrt(6.0 / i)
        parts.append(rng.uniform(-lim, lim, size=o * i))
        parts.append(np.zeros(o))
    return np.concatenate(parts).astype(np.float32)


def _blob(x, bins=12):
    x = np.clip(x, 0.0, 1.0)
    centers = np.arange(bins) + 0.5
    return np.maximum(0.0, 1.0 - np.abs(x[..., None] * bins - centers))


def _angles(d):
    theta = np.arccos(np.clip(d[..., 2], -1.0, 1.0)) / np.pi
    phi = (np.arctan2(d[..., 1], d[..., 0]) + np.pi) / (2 * np.pi)
    return theta, phi


def encode(pos01, n, wo):
    """pos01: (B,3) position already normalised to [0,1]^3; n, wo: (B,3) unit vectors."""
    B = pos01.shape[0]
    f = np.zeros((B, IN))
    f[:, 0:36] = _blob(pos01).reshape(B, 36)
    t, p = _angles(n)
    f[:, 36:48] = _blob(t)
    f[:, 48:60] = _blob(p)
    t, p = _angles(wo)
    f[:, 60:72] = _blob(t)
    f[:, 72:84] = _blob(p)
    f[:, 84] = 1.0
    return f


def forward(params, x, keep=False):
    layers = unpack(np.asarray(params, dtype=np.float64))
    acts = [x]
    h = x
    for li, (W, b) in enumerate(layers):
        z = h @ W.T + b
        h = np.maximum(z, 0.0) if li < len(layers) - 1 else z
        acts.append(h)
    return (h, acts) if keep else h


def mixture(y):
    """raw outputs (B, 48) -> weights (B,8), means (B,8,3), kappa (B,8) and intermediates."""
    r = y[:, :40].reshape(-1, LOBES, 5)
    logits = r[:, :, 0]
    logits = logits - logits.max(axis=1, keepdims=True)
    e = np.exp(logits)
    pi = e / e.sum(axis=1, keepdims=True)
    v = r[:, :, 1:4]
    vn = np.linalg.norm(v, axis=2, keepdims=True)
    mu = np.where(vn > 1e-12, v / np.maximum(vn, 1e-30), np.array([0.0, 0.0, 1.0]))
    raw = r[:, :, 4]
    sp = np.logaddexp(0.0, raw)
    kappa = np.minimum(sp + KAPPA_MIN, KAPPA_MAX)
    return pi, mu, kappa, vn, raw


def vmf(mu, kappa, w):
    c = kappa / (2 * np.pi * (-np.expm1(-2 * kappa)))
    return c * np.exp(kappa * (np.einsum("bkc,bc->bk", mu, w) - 1.0))


def pdf(y, w):
    pi, mu, kappa, _, _ = mixture(y)
    return (pi * vmf(mu, kappa, w)).sum(axis=1)


def loss_and_grad_y(y, wi, weight):
    """Returns (loss, dL/dy (B,48))."""
    B = y.shape[0]
    pi, mu, kappa, vn, raw = mixture(y)
    comp = vmf(mu, kappa, wi)                       # (B,8)
    q = (pi * comp).sum(axis=1)                     # (B,)
    mw = weight.mean()
    g = -(weight / (mw if mw > 0 else 1.0)) / B     # dL/dlog q
    loss = float((g * np.log(np.maximum(q, 1e-30))).sum())
    resp = pi * comp / np.maximum(q, 1e-30)[:, None]
    dlogit = resp - pi
    mudotw = np.einsum("bkc,bc->bk", mu, wi)
    dlogk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (mudotw - 1.0)
    dkappa = resp * dlogk
    sig = 1.0 / (1.0 + np.exp(-raw))
    dkraw = dkappa * sig * ((np.logaddexp(0.0, raw) + KAPPA_MIN) < KAPPA_MAX)
    dmu = (resp * kappa)[:, :, None] * (wi[:, None, :] - mudotw[:, :, None] * mu)
    dv = dmu / np.maximum(vn, 1e-30)
    dy = np.zeros_like(y)
    r = dy[:, :40].reshape(-1, LOBES, 5)
    r[:, :, 0] = dlogit * g[:, None]
    r[:, :, 1:4] = dv * g[:, None, None]
    r[:, :, 4] = dkraw * g[:, None]
    dy[:, :40] = r.reshape(B, 40)
    return loss, dy


def backward(params, acts, dy):
    layers = unpack(np.asarray(params, dtype=np.float64))
    grads = []
    d = dy
    for li in range(len(layers) - 1, -1, -1):
        W, b = layers[li]
        h_in = acts[li]
        grads.append((d.T @ h_in, d.sum(axis=0)))
        d = d @ W
        if li > 0:
            d = d * (acts[li] > 0)
    grads.reverse()
    return np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])


def train_step(params, m, v, t, x, wi, weight, lr):
    y, acts = forward(params, x, keep=True)
    loss, dy = loss_and_grad_y(y, wi, weight)
    g = backward(params, acts, dy)
    m = BETA1 * m + (1 - BETA1) * g
    v = BETA2 * v + (1 - BETA2) * g * g
    mh = m / (1 - BETA1 ** t)
    vh = v / (1 - BETA2 ** t)
    params = params - lr * mh / (np.sqrt(vh) + EPS)
    return params, m, v, loss, g


def sample(y, u_lobe, u1, u2):
    """Mixture sampling: lobe by the weights' CDF, then the vMF lobe (Jakob's inversion)."""
    pi, mu, kappa, _, _ = mixture(y)
    cdf = np.cumsum(pi, axis=1)
    k = np.minimum((cdf < u_lobe[:, None]).sum(axis=1), LOBES - 1)
    m = mu[np.arange(len(k)), k]
    kk = kappa[np.arange(len(k)), k]
    wz = 1.0 + np.log(u1 + (1.0 - u1) * np.exp(-2.0 * kk)) / kk
    r = np.sqrt(np.maximum(0.0, 1.0 - wz * wz))
    phi = 2 * np.pi * u2
    local = np.stack([r * np.cos(phi), r * np.sin(phi), wz], axis=1)
    # frame around m
    sign = np.where(m[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sign + m[:, 2])
    b = m[:, 0] * m[:, 1] * a
    t = np.stack([1 + sign * m[:, 0] ** 2 * a, sign * b, -sign * m[:, 0]], axis=1)
    bb = np.stack([b, sign + m[:, 1] ** 2 * a, -m[:, 1]], axis=1)
    return local[:, :1] * t + local[:, 1:2] * bb + local[:, 2:3] * m
