"""Seeded samples for the policy-network tests: 16 features, 4 classes from
a fixed nonlinear rule (so that a trained network can be scored)."""
import numpy as np


def mlp_samples(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 16)).astype(np.float32)
    s = x[:, 0] + 0.5 * x[:, 1] * x[:, 2]
    y = np.zeros(n, np.uint8)
    y[s > 0.8] = 1
    y[(s > 0.8) & (x[:, 3] > 0.3)] = 2
    y[x[:, 4] < -1.0] = 3
    return x, y


def mlp_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(64 * 16 + 64 + 64 * 64 + 64 + 3 * 64 + 3, np.float32)
    o = 0
    for rows, cols in ((64, 16), (64, 0), (64, 64), (64, 0), (3, 64), (3, 0)):
        k = rows * max(cols, 1)
        fan = cols if cols else 1
        p[o:o + k] = rng.normal(0, scale * np.sqrt(2.0 / fan) if cols else 0.1, k)
        o += k
    return p
