"""The CPU restatement of the learned-radius model (oracle/pg_mlp_oracle.py):
its gradient formulas against finite differences, BF16 rounding, Adam, features."""

import numpy as np

from oracle import pg_mlp_oracle as M


def _setup(seed=0, b=40):
    rng = np.random.default_rng(seed)
    params = rng.normal(0, 0.3, M.NPARAM)
    x = rng.normal(0, 1, (b, 16))
    t = rng.normal(0, 1, (b, 2))
    sw = (rng.random(b) > 0.2).astype(np.float64)
    return rng, params, x, t, sw, np.zeros(16), np.ones(16), np.zeros(2), np.ones(2)


def test_gradient_matches_finite_differences():
    rng, params, x, t, sw, mean, scale, tmean, tscale = _setup()
    loss, g = M.loss_and_grads(x, t, sw, params, mean, scale, tmean, tscale, rounding=False)
    idx = rng.choice(M.NPARAM, 60, replace=False)
    h = 1e-6
    for k in idx:
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        l1, _ = M.loss_and_grads(x, t, sw, p1, mean, scale, tmean, tscale, rounding=False)
        l2, _ = M.loss_and_grads(x, t, sw, p2, mean, scale, tmean, tscale, rounding=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, g[k])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, -3.14159, 0.0, 1.01171875], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 and r[6] == 1.015625  # ties to even
    assert r[3] == 1.0078125 and abs(r[4] + 3.140625) < 1e-7 and r[5] == 0.0
    assert (M.bf16(r) == r).all()


def test_rounded_gradient_close_to_exact():
    _, params, x, t, sw, mean, scale, tmean, tscale = _setup(1, 200)
    _, g0 = M.loss_and_grads(x, t, sw, params, mean, scale, tmean, tscale, rounding=False)
    _, g1 = M.loss_and_grads(x, t, sw, params, mean, scale, tmean, tscale, rounding=True)
    assert np.linalg.norm(g1 - g0) <= 0.05 * np.linalg.norm(g0)


def test_adam_step():
    p, g = np.array([1.0, -2.0]), np.array([0.5, -0.25])
    p1, m, v = M.adam(p, g, np.zeros(2), np.zeros(2), 1, 0.1)
    assert np.allclose(p1, p - 0.1 * np.sign(g), atol=1e-6)  # first step: lr * sign(g)


def test_features_scale_invariant_and_shapes():
    rng = np.random.default_rng(3)
    pts = rng.random((300, 3)).astype(np.float32)
    order = np.argsort(pts[:, 0], kind="stable")
    f1 = M.features(pts[order], None, np.array([0, 300]))
    f2 = M.features((pts[order] * 4.0).astype(np.float32), None, np.array([0, 300]))
    assert f1.shape == (300, 16)
    assert np.allclose(f1[:, :8].sum(1), 0.0, atol=1e-9)  # log distances relative to their mean
    assert np.allclose(f1, f2, atol=1e-5)                  # every feature is scale free
    one = M.features(pts[:1], None, np.array([0, 1]))
    assert (one == 0).all()
