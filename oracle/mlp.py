"""Float64 numpy restatement of the gear-selector MLP (12 -> 64 -> 64 -> 4,
exact-erf GELU, softmax cross-entropy) and its gradients — TEST
INFRASTRUCTURE ONLY: it checks the hand-written training kernels
(jb_gear_train_grad) and the fused inference (jb_gear_select).

Parameter vector layout: W1[64][12] b1[64] W2[64][64] b2[64] W3[4][64] b3[4].
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (64, 12)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (4, 64)),
                        ("b3", (4,))):
        k = int(np.prod(shape))
        out[name] = w[o:o + k].reshape(shape)
        o += k
    return out


def gelu(x):
    return 0.5 * x * (1 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


def forward(w, X):
    p = unpack(w)
    z1 = X @ p["W1"].T + p["b1"]
    h1 = gelu(z1)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = gelu(z2)
    o = h2 @ p["W3"].T + p["b3"]
    return z1, h1, z2, h2, o


def loss_and_grad(w, X, labels):
    """Summed (not averaged) softmax cross-entropy and its parameter gradient."""
    X = np.asarray(X, np.float64)
    p = unpack(w)
    z1, h1, z2, h2, o = forward(w, X)
    o = o - o.max(1, keepdims=True)
    pr = np.exp(o)
    pr /= pr.sum(1, keepdims=True)
    n = X.shape[0]
    loss = -np.log(np.maximum(pr[np.arange(n), labels], 1e-300)).sum()
    d3 = pr.copy()
    d3[np.arange(n), labels] -= 1.0
    d2 = (d3 @ p["W3"]) * gelu_d(z2)
    d1 = (d2 @ p["W2"]) * gelu_d(z1)
    g = np.concatenate([(d1.T @ X).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0), (d3.T @ h2).ravel(),
                        d3.sum(0)])
    return loss, g
