"""Checks of the float64 guiding model (oracle/guide_ref.py) on the CPU: the analytic gradient against
central finite differences, the mixture density integrating to one, and the mixture sampler drawing
from that density.  These pin the checker that the GPU guiding tests compare against."""
import numpy as np

import guide_ref as G


def _records(rng, n):
    pos = rng.uniform(0, 1, (n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    w = rng.exponential(1.0, n)
    return pos, nrm, wo, wi, w


def _loss(params, x, wi, w):
    y = G.forward(params, x)
    return G.loss_and_grad_y(y, wi, w)[0]


def test_param_count():
    assert G.param_count() == 96 * 64 + 64 + 3 * (64 * 64 + 64) + 64 * 48 + 48


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    params = G.init_params(7).astype(np.float64) * 0.5
    params += rng.normal(0, 0.01, params.shape)  # nonzero biases
    pos, nrm, wo, wi, w = _records(rng, 24)
    x = G.encode(pos, nrm, wo)
    y, acts = G.forward(params, x, keep=True)
    _, dy = G.loss_and_grad_y(y, wi, w)
    g = G.backward(params, acts, dy)
    idx = rng.choice(len(params), 60, replace=False)
    # include the last layer's concentration and logit rows
    idx = np.concatenate([idx, len(params) - 48 - np.arange(1, 6)])
    h = 1e-6
    for k in idx:
        p1 = params.copy()
        p1[k] += h
        p0 = params.copy()
        p0[k] -= h
        fd = (_loss(p1, x, wi, w) - _loss(p0, x, wi, w)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, g[k])


def test_mixture_density_integrates_to_one():
    rng = np.random.default_rng(4)
    y = rng.normal(0, 1.0, (3, 48))
    # directions on a fine Fibonacci sphere
    m = 200000
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    for b in range(3):
        q = G.pdf(np.repeat(y[b:b + 1], m, axis=0), dirs)
        assert abs(q.mean() * 4 * np.pi - 1.0) < 2e-3


def test_sampler_draws_from_the_density():
    rng = np.random.default_rng(5)
    y = rng.normal(0, 1.0, (1, 48))
    y[:, 4:40:5] = -1.0  # moderate concentrations keep E[1/q] finite and well estimated
    n = 400000
    yy = np.repeat(y, n, axis=0)
    d = G.sample(yy, rng.uniform(0, 1, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n))
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-9)
    q = G.pdf(yy, d)
    # E_q[1/q] = the sphere's area
    est = np.mean(1.0 / q)
    assert abs(est / (4 * np.pi) - 1.0) < 0.03
    # and a test function's expectation against quadrature
    f = lambda v: np.exp(2 * v[:, 0]) * (1 + v[:, 2] ** 2)
    m = 200000
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    qd = G.pdf(np.repeat(y, m, axis=0), dirs)
    exact = np.mean(f(dirs) * qd) * 4 * np.pi
    assert abs(np.mean(f(d)) / exact - 1.0) < 0.01
