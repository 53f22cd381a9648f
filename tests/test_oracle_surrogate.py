"""The float64 surrogate oracle's gradients against central finite differences (CPU)."""

import numpy as np

from oracle import surrogate


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    sizes = [6, 5, 5, 4]
    weights = [rng.standard_normal((sizes[i + 1], sizes[i])) * 0.7 for i in range(3)]
    biases = [rng.standard_normal(sizes[i + 1]) * 0.1 for i in range(3)]
    x, target = rng.standard_normal((7, 6)), rng.standard_normal((7, 4))
    loss, dws, dbs = surrogate.gradients(x, target, weights, biases, valid=3)
    h = 1e-6
    for layer in range(3):
        for params, grads in ((weights, dws), (biases, dbs)):
            flat = params[layer].reshape(-1)
            for i in range(0, flat.size, 3):
                old = flat[i]
                flat[i] = old + h
                up = surrogate.gradients(x, target, weights, biases, 3)[0]
                flat[i] = old - h
                down = surrogate.gradients(x, target, weights, biases, 3)[0]
                flat[i] = old
                assert abs((up - down) / (2 * h) - grads[layer].reshape(-1)[i]) < 1e-7
