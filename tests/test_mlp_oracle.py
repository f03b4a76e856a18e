"""The MLP oracle pinned on the CPU: analytic gradient vs central finite
differences, the epoch order is a permutation, and Adam fits a toy target."""
import numpy as np

import mlp_oracle as M


def _toy(n=300, I=5, O=3, seed=0):
    r = np.random.default_rng(seed)
    x = r.normal(size=(n, I))
    t = np.stack([np.sin(x[:, 0]) + x[:, 1] ** 2, x[:, 2] * x[:, 3], np.abs(x[:, 4])], 1)[:, :O]
    m = (r.random((n, O)) < 0.6).astype(np.float64)
    return x, t, m


def test_gradient_matches_finite_differences():
    I, H, O = 5, 7, 3
    x, t, m = _toy(40, I, O)
    _, n = M.layout(I, H, O)
    p = np.random.default_rng(1).normal(scale=0.5, size=n)
    loss, g = M.loss_grad(p, x, t, m, I, H, O)
    eps = 1e-6
    num = np.zeros(n)
    for k in range(n):
        d = np.zeros(n)
        d[k] = eps
        num[k] = (M.loss_grad(p + d, x, t, m, I, H, O)[0] - M.loss_grad(p - d, x, t, m, I, H, O)[0]) / (2 * eps)
    assert np.allclose(g, num, rtol=1e-5, atol=1e-7)
    assert loss > 0


def test_epoch_order_is_a_permutation():
    for n in (1, 2, 3, 5, 64, 100, 1000):
        for e in range(3):
            o = M.epoch_order(n, 42, e)
            assert sorted(o) == list(range(n))
    assert M.epoch_order(100, 42, 0) != M.epoch_order(100, 42, 1)


def test_adam_fits_toy_target():
    I, H, O = 5, 16, 3
    x, t, m = _toy(400, I, O)
    _, n = M.layout(I, H, O)
    p0 = np.random.default_rng(2).normal(scale=0.3, size=n)
    l0 = M.loss_grad(p0, x, t, m, I, H, O)[0]
    p, last, _ = M.train(p0, x, t, m, I, H, O, epochs=40, batch=32, lr=3e-3, seed=3)
    l1 = M.loss_grad(p, x, t, m, I, H, O)[0]
    assert l1 < 0.3 * l0
