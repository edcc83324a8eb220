"""CPU reference of the learned con2prim guess network -- TEST INFRASTRUCTURE ONLY.

Forward and backward of the 4 -> 64 -> 64 -> 64 -> 1 ReLU MLP in FP64 numpy,
with the parameter layout of include/verona_b200.h (W[in][out]). `bf16=True`
rounds the tensor-core operands (features, h1, h2, weights) to bfloat16 as the
GPU does, so the forward can be compared tightly; gradients are compared
against the plain FP64 backward. The GPU kernels are tested against it; the
product never imports it.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 4, 64


def split(v):
    v = np.asarray(v, dtype=np.float64)
    o, out = 0, {}
    for name, shape in (("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
                        ("W3", (N_H, N_H)), ("b3", (N_H,)), ("w4", (N_H,)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = v[o:o + n].reshape(shape)
        o += n
    return out


def join(d):
    return np.concatenate([d[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4")])


def bf16(x):
    """Round float64 values to the nearest bfloat16 (ties to even), back as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def relu(z):
    return np.maximum(z, 0.0)


def drelu(z):
    return (z > 0.0).astype(np.float64)


def forward(params, x, bf=False):
    p = split(params)
    q = (lambda a: bf16(a)) if bf else (lambda a: a)
    z1 = q(x) @ q(p["W1"])
    h1 = relu(z1 + p["b1"])
    z2 = q(h1) @ q(p["W2"])
    h2 = relu(z2 + p["b2"])
    z3 = q(h2) @ q(p["W3"])
    h3 = relu(z3 + p["b3"])
    y = h3 @ p["w4"] + p["b4"][0]
    return y, (z1, h1, z2, h2, z3, h3)


def loss_and_grad(params, x, t):
    """Mean squared error of y against t and its gradient (FP64)."""
    p = split(params)
    y, (z1, h1, z2, h2, z3, h3) = forward(params, x)
    n = x.shape[0]
    r = y - t
    dy = 2.0 * r / n
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, p["w4"]) * drelu(z3 + p["b3"])
    g["W3"] = h2.T @ dz3
    g["b3"] = dz3.sum(0)
    dz2 = (dz3 @ p["W3"].T) * drelu(z2 + p["b2"])
    g["W2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"].T) * drelu(z1 + p["b1"])
    g["W1"] = x.T @ dz1
    g["b1"] = dz1.sum(0)
    return float(np.mean(r * r)), join(g)
