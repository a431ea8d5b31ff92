"""GPU policy network (tensor-core forward / backward / Adam) against the
oracle restatement with the same bf16 operand rounding.

Tolerances: logits 2e-3 absolute + 1e-2 relative (the tensor cores sum in
another order, which can move a hidden activation across a bf16 rounding
boundary); loss 1e-4 relative; gradients 5e-3 relative L2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as orc  # noqa: E402
from mlp_data import mlp_params, mlp_samples  # noqa: E402


@pytest.fixture(scope="module")
def policy_cls():
    from nprush_b200 import build
    build.build()
    from nprush_b200.policy import AdcPolicy
    return AdcPolicy


@pytest.mark.parametrize("n", [1, 1000, 128 * 150 + 17])
def test_forward_matches_oracle(policy_cls, n):
    x, _ = mlp_samples(n, 10 + n)
    p = mlp_params(11)
    pol = policy_cls(params=p)
    got = pol.logits(x).cpu().numpy()
    _, _, want = orc.mlp_grads(p, x, None, round_bf16=True)
    err = np.abs(got - want)
    assert np.all(err <= 2e-3 + 1e-2 * np.abs(want)), err.max()
    assert np.median(err) < 1e-4


@pytest.mark.parametrize("n", [1, 1000, 128 * 150 + 17])
def test_gradients_match_oracle(policy_cls, n):
    x, y = mlp_samples(n, 20 + n)
    p = mlp_params(21)
    cw = (1.0, 2.0, 1.5, 3.0)
    pol = policy_cls(params=p)
    g, loss = pol.grads(x, y, cw)
    gw, lw, _ = orc.mlp_grads(p, x, y, cw, round_bf16=True)
    assert abs(loss - lw) <= 1e-4 * abs(lw) + 1e-6
    assert np.linalg.norm(g - gw) / np.linalg.norm(gw) < 5e-3
    # and the exact (double) gradient is close too: bf16 operands are the only difference
    _, g64 = orc.mlp_loss_f64(p, x, y, cw, with_grads=True)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 5e-2


def test_training_learns_the_rule(policy_cls):
    x, y = mlp_samples(60000, 30)
    xt, yt = mlp_samples(10000, 31)
    pol = policy_cls(seed=5)
    base = (pol.logits(xt).cpu().numpy() is not None)
    lc, ac = pol.train(x, y, epochs=15, batch=4096, lr=3e-3, seed=1)
    assert lc[-1] < 0.5 * lc[0], lc
    z = pol.logits(xt).cpu().numpy()
    pred = np.argmax(np.c_[np.zeros(len(z)), z], axis=1)
    assert base and (pred == yt).mean() > 0.9, (pred == yt).mean()


def test_training_is_bit_reproducible(policy_cls):
    """Each block's gradient, loss and count go to its own row and the rows
    are summed in block order: two trainings from the same seeds give the
    same parameters and curves bit for bit."""
    x, y = mlp_samples(20000, 40)
    out = []
    for _ in range(2):
        pol = policy_cls(seed=9)
        lc, ac = pol.train(x, y, epochs=4, batch=4096, lr=3e-3, seed=2)
        out.append((pol.params(), np.asarray(lc), np.asarray(ac)))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
