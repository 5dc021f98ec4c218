"""The FP64 oracle of the learned proposal: its gradient against finite differences, and
properties of the feature encoding (CPU only)."""
import numpy as np

import proposal_ref as P


def _net(seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, P.N_PARAMS)
    p[P.O_W1:P.O_B1].reshape(P.HID, P.N_IN)[:, P.N_FEAT:] = 0.0
    return p


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _net(1)
    x = rng.normal(0, 1, (40, P.N_IN))
    x[:, P.N_FEAT:] = 0.0
    y = (rng.random(40) < 0.3).astype(np.float64)
    loss, g = P.loss_and_grad(p, x, y)
    idx = np.concatenate([rng.choice(P.N_PARAMS, 60, replace=False), [P.O_B4, P.O_W4, P.O_B1, P.O_W3 + 5]])
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        lp, _ = P.loss_and_grad(p + e, x, y)
        lm, _ = P.loss_and_grad(p - e, x, y)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_forward_agrees_with_loss_path():
    rng = np.random.default_rng(2)
    p = _net(2)
    x = rng.normal(0, 1, (16, P.N_IN))
    z = P.forward(p, x)
    y = np.ones(16)
    loss, _ = P.loss_and_grad(p, x, y)
    assert np.isclose(loss, np.mean(np.log1p(np.exp(-z))))


def test_features_encode_midpoints():
    rng = np.random.default_rng(3)
    n = 50
    dims = (64, 64, 64)
    o = rng.uniform(-60, 120, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    near = rng.uniform(0, 50, n)
    far = near + rng.uniform(1, 80, n)
    f = P.features(*o.T, *d.T, near, far, dims)
    assert f.shape == (n, P.SEG, P.N_IN)
    assert not f[:, :, P.N_FEAT:].any()
    for k in range(4):
        for ax in range(3):
            s, c = f[:, :, 3 + 6 * k + 2 * ax], f[:, :, 4 + 6 * k + 2 * ax]
            assert np.allclose(s * s + c * c, 1.0)
    # the midpoint of segment s lies at near + (s + 0.5)(far - near) / 32 along the ray
    t = near[:, None] + (np.arange(P.SEG) + 0.5) * (far - near)[:, None] / P.SEG
    x = (o[:, None, :] + t[:, :, None] * d[:, None, :]) * (2.0 / 63) - 1
    assert np.allclose(f[:, :, :3], x)
    assert np.allclose(f[:, :, 27:30], d[:, None, :])
