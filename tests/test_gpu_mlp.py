"""The selector MLP's CUDA kernels vs the float64 oracle: forward outputs,
loss + gradient (the gradient check), and whole Adam training runs."""
import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu

DIMS = [(4, 8, 2), (9, 32, 4), (16, 64, 8), (1, 1, 1)]


def _data(n, I, O, seed):
    r = np.random.default_rng(seed)
    x = r.normal(size=(n, I)).astype(np.float32)
    t = r.normal(size=(n, O)).astype(np.float32)
    m = (r.random((n, O)) < 0.5).astype(np.float32)
    m[0, 0] = 1.0
    return x, t, m


@pytest.mark.parametrize("dims", DIMS)
def test_forward_matches_oracle(gpu_lib, dims):
    I, H, O = dims
    net = gpu_lib.Net(I, H, O, seed=11)
    x, _, _ = _data(300, I, O, 1)
    y = net.forward(x)
    want = M.forward(net.params(), x, I, H, O)
    assert np.allclose(y, want, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("n", [1, 63, 64, 65, 500])
def test_gradient_matches_oracle(gpu_lib, dims, n):
    I, H, O = dims
    net = gpu_lib.Net(I, H, O, seed=5 + n)
    x, t, m = _data(n, I, O, n)
    loss, g = net.loss_grad(x, t, m)
    lo, go = M.loss_grad(net.params(), x, t, m, I, H, O)
    assert abs(loss - lo) <= 1e-5 * max(1.0, abs(lo))
    scale = max(1.0, float(np.abs(go).max()))
    assert np.allclose(g, go, rtol=1e-4, atol=1e-5 * scale)


@pytest.mark.parametrize("dims", [(6, 16, 3), (16, 64, 8)])
def test_training_matches_oracle(gpu_lib, dims):
    I, H, O = dims
    net = gpu_lib.Net(I, H, O, seed=3)
    x, t, m = _data(257, I, O, 9)
    p0 = net.params().astype(np.float64)
    loss = net.train(x, t, m, epochs=3, batch=32, lr=1e-3, seed=21)
    p_ref, loss_ref, _ = M.train(p0, x, t, m, I, H, O, epochs=3, batch=32, lr=1e-3, seed=21)
    # fp32 vs fp64: Adam normalises each step by sqrt(v), so a parameter whose
    # gradient is ~0 may step +-lr on either side; nearly all must agree tightly
    # and none may drift by more than the 27 steps' worth of lr
    diff = np.abs(net.params() - p_ref)
    close = diff <= 1e-4 + 1e-3 * np.abs(p_ref)
    assert close.mean() >= 0.98, close.mean()
    assert diff.max() <= 2 * 27 * 1e-3
    assert abs(loss - loss_ref) <= 1e-3 * max(1.0, abs(loss_ref))
    # training continues from the stored Adam state
    net.train(x, t, m, epochs=2, batch=32, lr=1e-3, seed=22)


def test_training_fits_a_function(gpu_lib):
    I, H, O = 5, 32, 2
    r = np.random.default_rng(4)
    x = r.uniform(-1, 1, size=(2000, I)).astype(np.float32)
    t = np.stack([x[:, 0] * x[:, 1] + np.sin(3 * x[:, 2]), np.maximum(x[:, 3], x[:, 4])], 1).astype(np.float32)
    m = np.ones_like(t)
    net = gpu_lib.Net(I, H, O, seed=8)
    l0, _ = net.loss_grad(x, t, m)
    net.train(x, t, m, epochs=60, batch=64, lr=3e-3, seed=1)
    l1, _ = net.loss_grad(x, t, m)
    assert l1 < 0.1 * l0
