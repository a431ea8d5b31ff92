"""What the trained ADC policy gains over the plain threshold rule, on a
small seeded scene (20k-Gaussian student, 30k teacher, 256 x 256, 16
cameras, 4 views per step, 1200 steps, ADC every 100 from step 300): the
policy is trained on hindsight-labelled decisions logged from two plain runs
on other seeds, then both rules train the held-out scene.  Deterministic
mode makes each training run reproducible, and the policy's training is too
(its gradients are summed in a fixed order).  Checked: the learned rule ends
with no more Gaussians than the plain one (1% slack) and no worse PSNR (0.2 dB
slack).  At this scale the two rules differ by less than a change of the
scene or of the policy's seeds moves them (measured: 41421 vs 41402
Gaussians and 38.74 vs 38.63 dB; with earlier kernel versions 41302 vs 41402
and 39.05 vs 38.63 dB, 41411 vs 41402 and 38.61 vs 38.63 dB), so no strict gain is
asserted; the 30k-step comparison at 200k Gaussians, 800x800, is where the policy's effect
shows."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_learned_adc_keeps_psnr_with_fewer_gaussians():
    from nprush_b200 import build
    build.build()
    from nprush_b200.learned_adc import AdcLog, hindsight_labels, logging_adc_fn, policy_adc_fn
    from nprush_b200.policy import AdcPolicy
    from nprush_b200.train import AdcSchedule, teacher_scene, evaluate_psnr, fit

    adc = AdcSchedule(every=100, start=300, stop=1200)
    steps, views = 1200, 4

    def run(seed, adc_fn):
        vp, vpi, tg, st = teacher_scene(0, 20_000, 30_000, 256, 256, n_cams=16, sh_degree=1, capacity=60_000,
                                        student_seed=seed, teacher_seed=seed + 1000)
        st.set_deterministic(True)
        st.assign_ids(0)
        r = fit(st, vp, vpi, steps, views=views, seed=seed, adc=adc, mode="batched", adc_fn=adc_fn)
        psnr = float(np.mean(evaluate_psnr(st, vp, vpi, views=views)))
        st.close()
        return r, psnr

    log = AdcLog(samples_per_event=5000, seed=1)
    for s in (201, 202):
        run(s, logging_adc_fn(log, adc))
    X, y = hindsight_labels(log, horizon=3)
    assert (y == 3).sum() > 0 and (y == 0).sum() > 0
    pol = AdcPolicy(seed=7)
    lc, ac = pol.train(X, y, epochs=20, batch=4096, lr=2e-3, seed=3)
    assert lc[-1] < lc[0] and ac[-1] > 0.9
    plain, p_psnr = run(203, None)
    learned, l_psnr = run(203, policy_adc_fn(pol, adc))
    print(f"plain: {plain.count} Gaussians, {p_psnr:.2f} dB; learned: {learned.count} Gaussians, {l_psnr:.2f} dB")
    assert learned.count <= 1.01 * plain.count
    assert l_psnr > p_psnr - 0.2
