"""FP64 CPU restatement of the surrogate network (forward and backpropagation),
the checker of the tensor-core training kernels. Parameter layout as in
include/bbkde.h (bbkde_surrogate_num_params)."""
from __future__ import annotations

import numpy as np

H = 128
OFF = {}
_o = 0
for _name, _size in [("W1", H * 2), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H),
                     ("b3", H), ("w4", H), ("b4", 1)]:
    OFF[_name] = (_o, _size)
    _o += _size
N_PARAMS = _o


def unpack(p):
    g = {k: np.asarray(p[o:o + s], dtype=np.float64) for k, (o, s) in OFF.items()}
    g["W1"] = g["W1"].reshape(H, 2)
    g["W2"] = g["W2"].reshape(H, H)
    g["W3"] = g["W3"].reshape(H, H)
    return g


def pack(g):
    out = np.zeros(N_PARAMS)
    for k, (o, s) in OFF.items():
        out[o:o + s] = np.asarray(g[k]).ravel()
    return out


def bf16(a):
    """Round float64 values to bfloat16 (nearest even) and back."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, xin, emulate_bf16=False, bf16_weights=None):
    """xin: (n, 2) normalised inputs. emulate_bf16 rounds the hidden weights and the
    activations feeding the tensor-core layers to BF16; bf16_weights (default: the
    same) rounds only the weights. Returns (y, cache)."""
    g = unpack(p)
    q = bf16 if emulate_bf16 else (lambda a: a)
    qw = bf16 if (emulate_bf16 if bf16_weights is None else bf16_weights) else (lambda a: a)
    W2, W3 = qw(g["W2"]), qw(g["W3"])
    z1 = xin @ g["W1"].T + g["b1"]
    a1 = silu(z1)
    z2 = q(a1) @ W2.T + g["b2"]
    a2 = silu(z2)
    z3 = q(a2) @ W3.T + g["b3"]
    a3 = silu(z3)
    y = a3 @ g["w4"] + g["b4"][0]
    return y, dict(z1=z1, a1=q(a1), z2=z2, a2=q(a2), z3=z3, a3=a3, W2=W2, W3=W3, g=g)


def loss_and_grad(p, xin, t, emulate_bf16=False):
    """Mean squared error over the n rows and its gradient (float64)."""
    n = xin.shape[0]
    y, c = forward(p, xin, emulate_bf16)
    e = y - t
    loss = np.mean(e * e)
    dy = 2.0 * e / n
    g = c["g"]
    grads = {"w4": c["a3"].T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, g["w4"]) * silu_grad(c["z3"])
    grads["W3"] = dz3.T @ c["a2"]
    grads["b3"] = dz3.sum(0)
    dz2 = (dz3 @ c["W3"]) * silu_grad(c["z2"])
    grads["W2"] = dz2.T @ c["a1"]
    grads["b2"] = dz2.sum(0)
    dz1 = (dz2 @ c["W2"]) * silu_grad(c["z1"])
    grads["W1"] = dz1.T @ xin
    grads["b1"] = dz1.sum(0)
    return loss, pack(grads)


def loss_and_grad_tc(p, xin, t):
    """Mean squared error and its gradient with the rounding points of the
    tcgen05 training step (k_mlp_train_tc): BF16 hidden weights and BF16
    activations and output gradients as the operands of the four 128 x 128
    products, everything else (pre-activations, input gradients, bias and vector
    gradients, the first and last layer) unrounded."""
    n = xin.shape[0]
    g = unpack(p)
    W2, W3 = bf16(g["W2"]), bf16(g["W3"])
    z1 = xin @ g["W1"].T + g["b1"]
    a1 = bf16(silu(z1))
    z2 = a1 @ W2.T + g["b2"]
    a2 = bf16(silu(z2))
    z3 = a2 @ W3.T + g["b3"]
    a3 = silu(z3)
    y = a3 @ g["w4"] + g["b4"][0]
    e = y - t
    loss = np.mean(e * e)
    dy = 2.0 * e / n
    grads = {"w4": a3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, g["w4"]) * silu_grad(z3)
    grads["b3"] = dz3.sum(0)
    dZ3 = bf16(dz3)
    grads["W3"] = dZ3.T @ a2
    dz2 = (dZ3 @ W3) * silu_grad(z2)
    grads["b2"] = dz2.sum(0)
    dZ2 = bf16(dz2)
    grads["W2"] = dZ2.T @ a1
    dz1 = (dZ2 @ W2) * silu_grad(z1)
    grads["W1"] = dz1.T @ xin
    grads["b1"] = dz1.sum(0)
    return loss, pack(grads)
