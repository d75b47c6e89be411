"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the Johnson-Cook surrogate MLP
(4 -> 64 -> 64 -> 64 -> 1, SiLU) and of its mean-squared-error gradient, the checker of
the GPU training kernels.  Parameter layout as libsph_b200's sph_mlp_* entry points:
W1[64][4], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[64], b4.
"""
from __future__ import annotations

import numpy as np

H, NIN = 64, 4
SIZES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
         ("b3", (H,)), ("W4", (H,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = w[o:o + k].reshape(shape)
        o += k
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], dtype=np.float64).ravel() for name, _ in SIZES])


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(w, X):
    p = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ p["W1"].T + p["b1"]
    z2 = silu(z1) @ p["W2"].T + p["b2"]
    z3 = silu(z2) @ p["W3"].T + p["b3"]
    y = silu(z3) @ p["W4"] + p["b4"][0]
    return y, (X, z1, z2, z3)


def loss_and_grad(w, X, T):
    """Mean squared error over the rows and its gradient with respect to w."""
    p = unpack(w)
    y, (X, z1, z2, z3) = forward(w, X)
    n = len(y)
    e = y - np.asarray(T, dtype=np.float64)
    dy = 2.0 * e / n
    g = {"b4": np.array([dy.sum()]), "W4": silu(z3).T @ dy}
    d3 = np.outer(dy, p["W4"]) * silu_grad(z3)
    g["b3"], g["W3"] = d3.sum(0), d3.T @ silu(z2)
    d2 = (d3 @ p["W3"]) * silu_grad(z2)
    g["b2"], g["W2"] = d2.sum(0), d2.T @ silu(z1)
    d1 = (d2 @ p["W2"]) * silu_grad(z1)
    g["b1"], g["W1"] = d1.sum(0), d1.T @ X
    return float((e * e).mean()), pack(g)
