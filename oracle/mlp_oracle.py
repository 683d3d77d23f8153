"""CPU oracle of the surrogate ensemble (test infrastructure only): numpy float64 forward
and backward passes of the MLP with the BF16 rounding points of the device kernels
(weights, activations and pre-activation gradients stored as BF16; products accumulated
in high precision), and the Adam update.

Layer l computes Z_l = A_{l-1} W_l^T + b_l, A_l = bf16(GELU(Z_l)) (the last layer is linear);
the loss is the mean squared error over the real outputs.
"""
import math

import numpy as np


def bf16(x):
    """Round to BF16 (nearest, ties to even), returned as float32 values."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def rnd(x):
    """The device's storage rounding: to float32, then to BF16."""
    return bf16(np.asarray(x, np.float32))


def bf16_bits(x):
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(h):
    return (np.asarray(h, np.uint16).astype(np.uint32) << 16).view(np.float32)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def gemm(A, B, bias=None, act=False):
    """Z = A B^T (+ bias) in float64 from BF16-valued operands; returns (Z, bf16(act(Z)))."""
    z = A.astype(np.float64) @ B.astype(np.float64).T
    if bias is not None:
        z = z + bias.astype(np.float64)
    a = gelu(z) if act else z
    return z, rnd(a)


def forward(x, W, b):
    """x [M, K0] (BF16 values), W / b lists per layer; returns the pre-activations and
    BF16 activations of every layer (A[0] = x)."""
    A, Z = [x], []
    L = len(W)
    for l in range(L):
        z, a = gemm(A[-1], W[l], b[l], act=(l < L - 1))
        Z.append(z)
        A.append(a)
    return Z, A


def backward(Z, A, W, y_target, n_out):
    """Gradients of the mean squared error over the first n_out outputs (the device order:
    BF16 pre-activation gradients, FP64 products here)."""
    M = A[0].shape[0]
    L = len(W)
    y = Z[-1]
    g = np.zeros_like(y)
    g[:, :n_out] = 2.0 * (y[:, :n_out] - y_target) / (M * n_out)
    g = np.asarray(rnd(g), np.float64)
    dW, db = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        dW[l] = g.T @ A[l].astype(np.float64)
        db[l] = g.sum(axis=0)
        if l > 0:
            dA = g @ W[l].astype(np.float64)
            g = np.asarray(rnd(dA * gelu_grad(Z[l - 1])), np.float64)
    loss = float(((y[:, :n_out] - y_target) ** 2).mean())
    return dW, db, loss


def adam(w, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v
