"""Seeded ADC inputs: a scene with planted prune / clone / split candidates."""
import numpy as np

from gs_scenes import gs_scene


def adc_case(n, seed, deg=0):
    rng = np.random.default_rng(seed)
    p = gs_scene(n, seed, deg=deg)
    # about 10 % below the prune opacity (logit of 0.005 is -5.29)
    low = rng.random(n) < 0.1
    p[low, 10] = rng.uniform(-9.0, -5.5, low.sum())
    # half the scene large enough to split (max scale > 0.01 = e^-4.6)
    big = rng.random(n) < 0.5
    p[big, 3 + rng.integers(0, 3, big.sum())] = rng.uniform(-4.4, -2.0, big.sum())
    p[~big, 3:6] = rng.uniform(-7.0, -4.8, (int((~big).sum()), 3))
    m = rng.normal(0, 1e-3, p.shape).astype(np.float32)
    v = rng.random(p.shape).astype(np.float32) * 1e-6
    denom = rng.integers(0, 9, n).astype(np.float32)
    # about 30 % of the seen ones at or above the gradient threshold 2e-4
    avg = np.where(rng.random(n) < 0.3, rng.uniform(2.1e-4, 1e-3, n), rng.uniform(0.0, 1.9e-4, n))
    grad = (avg * denom).astype(np.float32)
    return p, m, v, grad, denom
