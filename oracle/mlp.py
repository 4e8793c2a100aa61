"""CPU oracle of the cooling network's forward and backward passes (TEST INFRASTRUCTURE).

The network (3 -> 64 -> 64 -> 64 SiLU -> 1) and its training loss have no counterpart in the
reference; this NumPy restatement checks the GPU kernels' gradients: forward with the weights
rounded to BF16 (round to nearest even, as the inference kernel stores them), mean squared error,
a sigmoid output (the network predicts logit f), and the straight-through backward pass in
float64.
"""

from __future__ import annotations

import numpy as np

H = 64
SIZES = [("W1", (H, 3)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
         ("W4", (1, H)), ("b4", (1,))]  # fmt: skip


def unpack(w):
    out, k = {}, 0
    for name, shape in SIZES:
        size = int(np.prod(shape))
        out[name] = np.asarray(w[k : k + size], np.float64).reshape(shape)
        k += size
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(w, X, Y):
    """(mean squared error, gradient (flat)) of the batch at weights w."""
    p = unpack(w)
    Wq = {k: bf16_round(p[k]).astype(np.float64) if k.startswith("W") else p[k] for k in p}
    X = np.asarray(X, np.float64)
    z1 = X @ Wq["W1"].T + Wq["b1"]
    a1 = silu(z1)
    z2 = a1 @ Wq["W2"].T + Wq["b2"]
    a2 = silu(z2)
    z3 = a2 @ Wq["W3"].T + Wq["b3"]
    a3 = silu(z3)
    y = 1.0 / (1.0 + np.exp(-(a3 @ Wq["W4"].T + Wq["b4"])))  # f = sigmoid(z4)
    d = y[:, 0] - np.asarray(Y, np.float64)
    B = len(X)
    loss = float(np.mean(d * d))
    dy = (2.0 * d * y[:, 0] * (1.0 - y[:, 0]) / B)[:, None]
    g = {"W4": dy.T @ a3, "b4": dy.sum(0)}
    dz3 = (dy @ Wq["W4"]) * dsilu(z3)
    g["W3"], g["b3"] = dz3.T @ a2, dz3.sum(0)
    dz2 = (dz3 @ Wq["W3"]) * dsilu(z2)
    g["W2"], g["b2"] = dz2.T @ a1, dz2.sum(0)
    dz1 = (dz2 @ Wq["W2"]) * dsilu(z1)
    g["W1"], g["b1"] = dz1.T @ X, dz1.sum(0)
    return loss, pack(g)


def predict(w, X):
    """Network output f (float64 arithmetic, BF16 weights)."""
    p = unpack(w)
    Wq = {k: bf16_round(p[k]).astype(np.float64) if k.startswith("W") else p[k] for k in p}
    a = np.asarray(X, np.float64)
    for i in (1, 2, 3):
        a = silu(a @ Wq[f"W{i}"].T + Wq[f"b{i}"])
    return 1.0 / (1.0 + np.exp(-(a @ Wq["W4"].T + Wq["b4"])[:, 0]))


def label(u, rho, dt, consts):
    """f = (u - u_new) / (u - u_floor) of the exact bremsstrahlung integrator (0 at the floor)."""
    from .cooling import brems_cool

    un = brems_cool(u, rho, dt, consts)
    d = np.asarray(u) - consts[3]
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(d > 0, (np.asarray(u) - un) / d, 0.0)
