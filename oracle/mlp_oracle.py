"""CPU oracle of the schedule selector's MLP (TEST INFRASTRUCTURE ONLY).

Only tests/ and __graft_entry__.smoke() use it, to check the CUDA kernels
behind gmpt_mlp_forward / gmpt_mlp_loss_grad / gmpt_mlp_train.  Float64
numpy restatement of the same network and training rule:

* parameters, flat: W1[H][I] b1[H] W2[H][H] b2[H] W3[O][H] b3[O];
  y = W3 relu(W2 relu(W1 x + b1) + b2) + b3;
* loss = sum(M * (y - T)^2) / sum(M) (masked mean squared error);
* Adam (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected), mini-batch loss
  normalised by the mini-batch's mask sum;
* epoch e visits positions j = 0 .. P-1 (P = next power of two >= n) as
  sample (a_e * j + b_e) mod P, skipping images >= n, a_e odd, a_e and b_e
  from splitmix64 of the seed and e.

The analytic gradient is itself pinned against central finite differences
in the tests.  There is no reference implementation of this component (the
reference has no runtime schedule selector), so this oracle is the spec.
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def layout(I: int, H: int, O: int):
    sizes = [("W1", (H, I)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
    out, at = {}, 0
    for name, shp in sizes:
        n = int(np.prod(shp))
        out[name] = (at, shp)
        at += n
    return out, at


def unpack(p, I, H, O):
    lay, _ = layout(I, H, O)
    return {k: np.asarray(p[a: a + int(np.prod(s))], dtype=np.float64).reshape(s) for k, (a, s) in lay.items()}


def pack(d, I, H, O):
    lay, n = layout(I, H, O)
    p = np.zeros(n, dtype=np.float64)
    for k, (a, s) in lay.items():
        p[a: a + int(np.prod(s))] = d[k].reshape(-1)
    return p


def forward(p, x, I, H, O):
    w = unpack(p, I, H, O)
    x = np.asarray(x, dtype=np.float64)
    a1 = np.maximum(x @ w["W1"].T + w["b1"], 0.0)
    a2 = np.maximum(a1 @ w["W2"].T + w["b2"], 0.0)
    return a2 @ w["W3"].T + w["b3"]


def loss_grad(p, x, t, m, I, H, O, norm=None):
    """Masked-MSE loss and its gradient w.r.t. the flat parameters."""
    w = unpack(p, I, H, O)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    z1 = x @ w["W1"].T + w["b1"]
    a1 = np.maximum(z1, 0.0)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = np.maximum(z2, 0.0)
    y = a2 @ w["W3"].T + w["b3"]
    if norm is None:
        s = m.sum()
        norm = 1.0 / s if s > 0 else 0.0
    r = y - t
    loss = norm * np.sum(m * r * r)
    dy = 2.0 * norm * m * r
    g = {"W3": dy.T @ a2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * (z2 > 0)
    g["W2"] = dz2.T @ a1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * (z1 > 0)
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return loss, pack(g, I, H, O)


def epoch_order(n: int, seed: int, epoch: int):
    P = 1
    while P < n:
        P <<= 1
    h = splitmix64(seed ^ ((0x632BE59BD9B4E019 * (epoch + 1)) & M64))
    a = (h | 1) & (P - 1)
    if a == 0:
        a = 1
    b = splitmix64(h) & (P - 1)
    out = []
    for j in range(P):
        idx = (a * j + b) & (P - 1)
        if idx < n:
            out.append(idx)
    return out


class Adam:
    def __init__(self, n_params: int):
        self.m = np.zeros(n_params)
        self.v = np.zeros(n_params)
        self.t = 0

    def step(self, p, g, lr):
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        mh = self.m / (1 - 0.9 ** self.t)
        vh = self.v / (1 - 0.999 ** self.t)
        return p - lr * mh / (np.sqrt(vh) + 1e-8)


def train(p, x, t, m, I, H, O, epochs, batch, lr, seed, adam: Adam | None = None):
    """Same visiting order and update rule as gmpt_mlp_train."""
    adam = adam or Adam(len(p))
    p = np.asarray(p, dtype=np.float64).copy()
    n = len(x)
    last = 0.0
    for e in range(epochs):
        order = epoch_order(n, seed, e)
        losses = []
        for s in range(0, n, batch):
            idx = order[s: s + batch]
            loss, g = loss_grad(p, x[idx], t[idx], m[idx], I, H, O)
            losses.append(loss)
            p = adam.step(p, g, lr)
        last = float(np.mean(losses)) if losses else 0.0
    return p, last, adam
