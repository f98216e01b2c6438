"""CPU ORACLE — test infrastructure only (checker of the surrogate MLP kernels).

float64 numpy restatement of the network the dtb_mlp_* kernels compute:
in -> H -> H -> 1, GELU(x) = x * Phi(x) (erf form), weights rounded to BF16
(round-to-nearest-even of the FP32 master, as the kernels use them), biases FP32,
loss = mean((y - t)^2).  Returns the loss and the gradient in the kernels' flat
parameter order W1, b1, W2, b2, W3, b3.
"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16_round(w: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w: np.ndarray, in_dim: int, H: int):
    o = 0
    W1 = w[o:o + H * in_dim].reshape(H, in_dim); o += H * in_dim
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    W3 = w[o:o + H]; o += H
    b3 = w[o:o + 1]
    return W1, b1, W2, b2, W3, b3


def forward_backward(w: np.ndarray, x: np.ndarray, t: np.ndarray, in_dim: int, H: int, round_weights: bool = True):
    W1, b1, W2, b2, W3, b3 = unpack(w.astype(np.float64), in_dim, H)
    if round_weights:
        W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    x = x.astype(np.float64)
    t = t.astype(np.float64)
    phi = lambda z: 0.5 * (1.0 + _erf(z / math.sqrt(2.0)))
    Z1 = x @ W1.T + b1
    H1 = Z1 * phi(Z1)
    Z2 = H1 @ W2.T + b2
    H2 = Z2 * phi(Z2)
    y = H2 @ W3 + b3[0]
    B = x.shape[0]
    loss = np.mean((y - t) ** 2)
    dy = 2.0 * (y - t) / B
    gelu_grad = lambda z: phi(z) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    dW3 = dy @ H2
    db3 = np.array([dy.sum()])
    dZ2 = np.outer(dy, W3) * gelu_grad(Z2)
    dW2 = dZ2.T @ H1
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * gelu_grad(Z1)
    dW1 = dZ1.T @ x
    db1 = dZ1.sum(0)
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, db3])
    return y, loss, grad
