"""FP64 CPU restatement of the scheduler network (TEST INFRASTRUCTURE ONLY).

Same layout as the engine (include/cgb200.h, CGB_POLICY_PARAMS):
W1[24][64] b1[64] W2[64][64] b2[64] W3[64][14] b3[14], ReLU after the two
hidden layers, loss = sum(mask * (Y - T)^2) / sum(mask).  Used to check the
GPU forward pass and the GPU gradient, and checked itself by central finite
differences.
"""
from __future__ import annotations

import numpy as np

F, H, O = 24, 64, 14
SIZES = [("W1", (F, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, O)), ("b3", (O,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, np.float64)
    a1 = X @ w["W1"] + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ w["W3"] + w["b3"]
    return y, (X, a1, h1, a2, h2)


def loss(p, X, T, M):
    y, _ = forward(p, X)
    M = np.asarray(M, np.float64)
    return float(np.sum(M * (y - T) ** 2) / np.sum(M))


def loss_grad(p, X, T, M):
    w = unpack(p)
    y, (X, a1, h1, a2, h2) = forward(p, X)
    M = np.asarray(M, np.float64)
    cnt = np.sum(M)
    dy = 2 * M * (y - np.asarray(T, np.float64)) / cnt
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    dh2 = (dy @ w["W3"].T) * (a2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ w["W2"].T) * (a1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return float(np.sum(M * (y - T) ** 2) / cnt), g


def finite_diff(p, X, T, M, idx, eps=1e-6):
    p = np.asarray(p, np.float64)
    out = []
    for i in idx:
        a = p.copy()
        b = p.copy()
        a[i] += eps
        b[i] -= eps
        out.append((loss(a, X, T, M) - loss(b, X, T, M)) / (2 * eps))
    return np.array(out)
