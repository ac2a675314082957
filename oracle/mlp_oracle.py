"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the learned closure's network
(myfvcomcode_b200/csrc/k_mlp.cu) -- forward pass, mean-squared error and its gradient --
used to check the CUDA training kernels' gradients.  Parameter layout as in the kernels:
W1 (64x8), b1 (64), W2 (64x64), b2 (64), W3 (3x64), b3 (3), concatenated.
"""
from __future__ import annotations

import math

import numpy as np

MI, MH, MO = 8, 64, 3
SIZES = [("W1", (MH, MI)), ("b1", (MH,)), ("W2", (MH, MH)), ("b2", (MH,)), ("W3", (MO, MH)), ("b3", (MO,))]
NPAR = sum(int(np.prod(s)) for _, s in SIZES)



def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


GC = math.sqrt(2.0 / math.pi)
GA = 0.044715


def gelu(z):
    """GELU in its tanh form, as the kernels use it."""
    return 0.5 * z * (1.0 + np.tanh(GC * (z + GA * z ** 3)))


def gelu_d(z):
    t = np.tanh(GC * (z + GA * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GC * (1.0 + 3.0 * GA * z * z)


def forward(p, x):
    w = unpack(p)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = gelu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = gelu(z2)
    return h2 @ w["W3"].T + w["b3"], (z1, h1, z2, h2)


def loss_grad(p, x, y):
    """Mean-squared error over all n*3 outputs and its gradient, in float64."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    w = unpack(p)
    out, (z1, h1, z2, h2) = forward(p, x)
    n = x.shape[0]
    e = out - y
    loss = float(np.mean(e * e))
    dy = 2.0 * e / (n * MO)
    g = {"W3": dy.T @ h2, "b3": dy.sum(axis=0)}
    dz2 = (dy @ w["W3"]) * gelu_d(z2)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(axis=0)
    dz1 = (dz2 @ w["W2"]) * gelu_d(z1)
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(axis=0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SIZES])


def bf16(a):
    """Round float values to the nearest-even bfloat16 (returned as float64)."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, x):
    """The tensor-core kernel's arithmetic: BF16 inputs, weights and hidden activations,
    products summed in (at least) FP32, biases and GELU in FP32."""
    w = unpack(p)
    a = bf16(x)
    z1 = a @ bf16(w["W1"]).T + w["b1"].astype(np.float32)
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(w["W2"]).T + w["b2"].astype(np.float32)
    h2 = bf16(gelu(z2))
    return h2 @ bf16(w["W3"]).T + w["b3"].astype(np.float32)
