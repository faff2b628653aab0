"""ORACLE — test infrastructure only (not product code).

FP64 numpy restatement of the settings network of saplibrary_b200/csrc/mlp.cu
(in -> h1 -> h2 -> out, ReLU hidden layers, mean softmax cross-entropy) with
its gradient in the same flat parameter layout (W1 [h1][in], b1, W2, b2,
W3, b3), the checker of the GPU forward and backward kernels.
"""
from __future__ import annotations

import numpy as np


def unpack(p: np.ndarray, shape):
    i, h1, h2, o = shape
    p = np.asarray(p, np.float64)
    sizes = [h1 * i, h1, h2 * h1, h2, o * h2, o]
    parts, k = [], 0
    for s in sizes:
        parts.append(p[k:k + s])
        k += s
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(h1, i), b1, W2.reshape(h2, h1), b2, W3.reshape(o, h2), b3


def forward(p, shape, X):
    W1, b1, W2, b2, W3, b3 = unpack(p, shape)
    X = np.asarray(X, np.float64)
    a1 = np.maximum(X @ W1.T + b1, 0.0)
    a2 = np.maximum(a1 @ W2.T + b2, 0.0)
    return a1, a2, a2 @ W3.T + b3


def loss_and_grad(p, shape, X, y):
    W1, b1, W2, b2, W3, b3 = unpack(p, shape)
    X = np.asarray(X, np.float64)
    a1, a2, z = forward(p, shape, X)
    B = X.shape[0]
    zs = z - z.max(axis=1, keepdims=True)
    lse = np.log(np.exp(zs).sum(axis=1, keepdims=True))
    logp = zs - lse
    loss = -logp[np.arange(B), y].mean()
    dz = np.exp(logp)
    dz[np.arange(B), y] -= 1.0
    dz /= B
    dW3, db3 = dz.T @ a2, dz.sum(axis=0)
    d2 = (dz @ W3) * (a2 > 0)
    dW2, db2 = d2.T @ a1, d2.sum(axis=0)
    d1 = (d2 @ W2) * (a1 > 0)
    dW1, db1 = d1.T @ X, d1.sum(axis=0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g
