"""CPU checks of the policy-network oracle: its analytic backward against
FP64 central differences, and its bf16-rounded mode close to exact."""
import numpy as np

import oracle as orc
from mlp_data import mlp_params, mlp_samples


def test_mlp_backward_matches_central_differences():
    x, y = mlp_samples(64, 1)
    p = mlp_params(2)
    cw = (1.0, 2.0, 0.5, 3.0)
    loss, g = orc.mlp_loss_f64(p, x, y, cw, with_grads=True)
    rng = np.random.default_rng(3)
    idx = rng.choice(p.size, 60, replace=False)
    for i in idx:
        h = 1e-4 * max(1.0, abs(float(p[i])))  # small enough to cross no ReLU kink
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        # the oracle reads fp32 parameters: step in fp32-representable amounts
        pp[i] += h
        pm[i] -= h
        hp = np.float32(pp[i]) - np.float32(p[i])
        hm = np.float32(p[i]) - np.float32(pm[i])
        lp = orc.mlp_loss_f64(pp.astype(np.float32), x, y, cw)
        lm = orc.mlp_loss_f64(pm.astype(np.float32), x, y, cw)
        cd = (lp - lm) / (float(hp) + float(hm))
        assert abs(cd - g[i]) <= 1e-5 + 1e-3 * abs(g[i]), (i, cd, g[i])


def test_mlp_bf16_mode_close_to_exact():
    x, y = mlp_samples(512, 4)
    p = mlp_params(5)
    g32, l32, z32 = orc.mlp_grads(p, x, y, round_bf16=False)
    gb, lb, zb = orc.mlp_grads(p, x, y, round_bf16=True)
    assert abs(lb - l32) < 2e-2 * abs(l32)
    assert np.linalg.norm(gb - g32) / np.linalg.norm(g32) < 3e-2
    np.testing.assert_allclose(zb, z32, atol=0.1 * np.abs(z32).max())
