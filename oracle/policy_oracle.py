"""ORACLE - test infrastructure only.

fp64 numpy restatement of the learned Delta policy network (12 -> 64 -> 64 -> 64 -> 16,
ReLU, softmax cross-entropy against soft targets), its gradient, and a
finite-difference check of that gradient. The network has no counterpart in the
reference; the CUDA kernels of pathfinding_gpu_b200/csrc/pfg_policy.cu are checked
against this file. Parameter layout (flat float32 image): w1[64x12] b1[64]
w2[64x64] b2[64] w3[64x64] b3[64] w4[16x64] b4[16] in_mean[12] in_scale[12].
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 12, 64, 16
SIZES = [("w1", (H, IN)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)), ("w3", (H, H)), ("b3", (H,)),
         ("w4", (OUT, H)), ("b4", (OUT,)), ("in_mean", (IN,)), ("in_scale", (IN,))]
NP = sum(int(np.prod(s)) for _, s in SIZES)


def unflatten(flat):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def flatten(p):
    return np.concatenate([np.asarray(p[name], np.float64).reshape(-1) for name, _ in SIZES])


def forward(flat, X):
    p = unflatten(flat)
    a0 = (np.asarray(X, np.float64) - p["in_mean"]) * p["in_scale"]
    z1 = a0 @ p["w1"].T + p["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(z2, 0)
    z3 = h2 @ p["w3"].T + p["b3"]
    h3 = np.maximum(z3, 0)
    z = h3 @ p["w4"].T + p["b4"]
    return z, (a0, h1, h2, h3)


def loss(flat, X, Y):
    z, _ = forward(flat, X)
    zmax = z.max(axis=1, keepdims=True)
    lse = zmax[:, 0] + np.log(np.exp(z - zmax).sum(axis=1))
    return float(np.mean(np.sum(np.asarray(Y, np.float64) * (lse[:, None] - z), axis=1)))


def grad(flat, X, Y):
    """Gradient of `loss` for every parameter (zero for the fixed normalisation)."""
    p = unflatten(flat)
    z, (a0, h1, h2, h3) = forward(flat, X)
    n = len(X)
    zmax = z.max(axis=1, keepdims=True)
    e = np.exp(z - zmax)
    pr = e / e.sum(axis=1, keepdims=True)
    dz = (pr - np.asarray(Y, np.float64)) / n
    g = {name: np.zeros(shape) for name, shape in SIZES}
    g["w4"] = dz.T @ h3
    g["b4"] = dz.sum(0)
    d3 = (dz @ p["w4"]) * (h3 > 0)
    g["w3"] = d3.T @ h2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ p["w3"]) * (h2 > 0)
    g["w2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ p["w2"]) * (h1 > 0)
    g["w1"] = d1.T @ a0
    g["b1"] = d1.sum(0)
    return flatten(g)


def predict(flat, X):
    z, _ = forward(flat, X)
    return np.argmax(z, axis=1)


def finite_difference(flat, X, Y, idx, eps=1e-6):
    f = np.asarray(flat, np.float64).copy()
    out = []
    for i in idx:
        a = f.copy()
        b = f.copy()
        a[i] += eps
        b[i] -= eps
        out.append((loss(a, X, Y) - loss(b, X, Y)) / (2 * eps))
    return np.asarray(out)
