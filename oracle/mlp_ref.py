"""CPU oracle for the cost model's MLP (TEST INFRASTRUCTURE ONLY).

float64 numpy restatement of the 16 -> 64 -> 64 -> 1 ReLU network of
compression_b200/csrc/mlp.cu, its mean-squared-error loss and the analytic
gradient, plus a central finite-difference gradient to check the analytic one.
Parameter layout: W1[16][64] | b1[64] | W2[64][64] | b2[64] | W3[64] | b3.
"""
from __future__ import annotations

import numpy as np

IN, H = 16, 64
SIZES = [IN * H, H, H * H, H, H, 1]
NP = sum(SIZES)


def unpack(p):
    p = np.asarray(p, np.float64)
    o = np.cumsum([0] + SIZES)
    return (p[o[0]:o[1]].reshape(IN, H), p[o[1]:o[2]], p[o[2]:o[3]].reshape(H, H), p[o[3]:o[4]],
            p[o[4]:o[5]], p[o[5]])


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    z1 = X @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def loss(p, X, y):
    o, _ = forward(p, X)
    return float(np.mean((o - y) ** 2))


def grad(p, X, y):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    o, (z1, h1, z2, h2) = forward(p, X)
    n = X.shape[0]
    d = 2.0 * (o - y) / n
    gW3 = h2.T @ d
    gb3 = np.array([d.sum()])
    dz2 = np.outer(d, W3) * (z2 > 0)
    gW2 = h1.T @ dz2
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2.T) * (z1 > 0)
    gW1 = X.T @ dz1
    gb1 = dz1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, gb3])


def fd_grad(p, X, y, idx, h=1e-6):
    """Central differences of the loss for the parameters listed in idx."""
    p = np.asarray(p, np.float64).copy()
    out = []
    for i in idx:
        a = p.copy()
        b = p.copy()
        a[i] += h
        b[i] -= h
        out.append((loss(a, X, y) - loss(b, X, y)) / (2 * h))
    return np.array(out)
