"""CPU restatement of the learned scheduler's network (test infrastructure
only: the gradient check of the CUDA training kernels and the reference for
their forward pass).

A 16-64-64-3 multilayer perceptron with ReLU, weight matrices rounded to
BF16 (round to nearest even) in the forward pass, FP32 biases, and the loss
L = (1/n) sum_r w[y_r] * CE(softmax(z_r), y_r).  The gradient with respect to
the FP32 master weights passes the BF16 rounding straight through, as the
CUDA kernels do.  Parameters are one flat array: W1[16][64], b1[64],
W2[64][64], b2[64], W3[64][3], b3[3].
"""
from __future__ import annotations

import numpy as np

N_PARAMS = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 3 + 3
_SPLITS = [(0, 1024, (16, 64)), (1024, 1088, (64,)), (1088, 5184, (64, 64)), (5184, 5248, (64,)),
           (5248, 5440, (64, 3)), (5440, 5443, (3,))]


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray, quantize: bool = True):
    parts = [np.asarray(p[a:b], dtype=np.float64).reshape(shape) for a, b, shape in _SPLITS]
    if quantize:
        for k in (0, 2, 4):
            parts[k] = bf16_round(np.asarray(p[_SPLITS[k][0]:_SPLITS[k][1]], np.float32)).astype(
                np.float64).reshape(_SPLITS[k][2])
    return parts


def forward(p, X, quantize=True):
    W1, b1, W2, b2, W3, b3 = unpack(p, quantize)
    X = np.asarray(X, np.float64)
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ W3 + b3
    return z, (X, h1, h2)


def loss_and_grad(p, X, y, class_weight=(1.0, 1.0, 1.0), quantize=True):
    W1, b1, W2, b2, W3, b3 = unpack(p, quantize)
    z, (X, h1, h2) = forward(p, X, quantize)
    y = np.asarray(y, np.int64)
    n = X.shape[0]
    w = np.asarray(class_weight, np.float64)[y] / n
    m = z.max(axis=1, keepdims=True)
    e = np.exp(z - m)
    s = e.sum(axis=1, keepdims=True)
    prob = e / s
    loss = float(np.sum(w * (np.log(s[:, 0]) + m[:, 0] - z[np.arange(n), y])))
    dz = prob.copy()
    dz[np.arange(n), y] -= 1.0
    dz *= w[:, None]
    gW3 = h2.T @ dz
    gb3 = dz.sum(0)
    dh2 = (dz @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
