"""CPU restatement of the learned scheduler's network (test infrastructure
only: the gradient check of the CUDA training kernels and the reference for
their forward pass).

A 16-64-64-3 multilayer perceptron with ReLU, FP32 biases, and the loss
L = (1/n) sum_r w[y_r] * CE(softmax(z_r), y_r).  Parameters are one flat
array: W1[16][64], b1[64], W2[64][64], b2[64], W3[64][3], b3[3].

With quantize=True the numerics are those of the CUDA kernels, which run the
products on the tensor cores (BF16 operands, FP32 accumulation): every
operand of a matrix product -- weight matrices, inputs, hidden activations,
and in the backward pass the errors at the logits and at both hidden layers
-- is rounded to BF16 (nearest even) as it enters the product; the ReLU masks
use the unrounded activations, bias gradients sum the rounded errors, and the
gradient with respect to the FP32 master weights passes the weights' BF16
rounding straight through.  With quantize=False everything stays FP64 (the
finite-difference check).
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


def _operand(a, quantize):
    """An operand of a matrix product: rounded to BF16 (through FP32) when quantize."""
    return bf16_round(np.asarray(a, np.float32)).astype(np.float64) if quantize else np.asarray(a, np.float64)


def forward(p, X, quantize=True):
    W1, b1, W2, b2, W3, b3 = unpack(p, quantize)
    Xq = _operand(X, quantize)
    a1 = Xq @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = _operand(h1, quantize) @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    z = _operand(h2, quantize) @ W3 + b3
    return z, (Xq, h1, h2)


def loss_and_grad(p, X, y, class_weight=(1.0, 1.0, 1.0), quantize=True):
    W1, b1, W2, b2, W3, b3 = unpack(p, quantize)
    z, (Xq, h1, h2) = forward(p, X, quantize)
    y = np.asarray(y, np.int64)
    n = Xq.shape[0]
    w = np.asarray(class_weight, np.float64)[y] / n
    m = z.max(axis=1, keepdims=True)
    e = np.exp(z - m)
    s = e.sum(axis=1, keepdims=True)
    prob = e / s
    loss = float(np.sum(w * (np.log(s[:, 0]) + m[:, 0] - z[np.arange(n), y])))
    dz = prob.copy()
    dz[np.arange(n), y] -= 1.0
    dz = _operand(dz * w[:, None], quantize)
    h1q, h2q = _operand(h1, quantize), _operand(h2, quantize)
    gW3 = h2q.T @ dz
    gb3 = dz.sum(0)
    dh2 = _operand((dz @ W3.T) * (h2 > 0), quantize)
    gW2 = h1q.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = _operand((dh2 @ W2.T) * (h1 > 0), quantize)
    gW1 = Xq.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
