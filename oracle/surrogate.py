"""NumPy float64 forward and backward of the surrogate MLP (TEST INFRASTRUCTURE ONLY: the checker
of the BF16 tensor-core training kernels).

The reference has no surrogate, so there is nothing of the reference's to restate; this is the
mathematics of the network the kernels implement: Z_l = Y_{l-1} W_l^T + b_l, Y_l = gelu(Z_l)
(tanh form) for the hidden layers, a linear output layer, and the mean squared error over the
first ``valid`` outputs, L = sum (out - target)^2 / (M valid), with its exact gradients.
"""

from __future__ import annotations

import numpy as np

_C = np.sqrt(2.0 / np.pi)
_A = 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(_C * (z + _A * z**3)))


def gelu_grad(z):
    t = np.tanh(_C * (z + _A * z**3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3.0 * _A * z * z)


def forward(x, weights, biases):
    """(pre-activations, activations, output) in float64."""

    zs, ys = [], [np.asarray(x, dtype=float)]
    for layer, (w, b) in enumerate(zip(weights, biases)):
        z = ys[-1] @ np.asarray(w, dtype=float).T + np.asarray(b, dtype=float)
        zs.append(z)
        ys.append(gelu(z) if layer < len(weights) - 1 else z)
    return zs, ys, ys[-1]


def gradients(x, target, weights, biases, valid: int):
    """Loss and (dW, db) per layer of the masked mean squared error."""

    zs, ys, out = forward(x, weights, biases)
    m = out.shape[0]
    diff = np.zeros_like(out)
    diff[:, :valid] = out[:, :valid] - np.asarray(target, dtype=float)[:, :valid]
    loss = float(np.sum(diff * diff) / (m * valid))
    g = 2.0 * diff / (m * valid)
    dws, dbs = [None] * len(weights), [None] * len(weights)
    for layer in range(len(weights) - 1, -1, -1):
        dws[layer] = g.T @ ys[layer]
        dbs[layer] = g.sum(axis=0)
        if layer > 0:
            g = (g @ np.asarray(weights[layer], dtype=float)) * gelu_grad(zs[layer - 1])
    return loss, dws, dbs
