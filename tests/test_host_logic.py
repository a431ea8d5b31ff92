"""CPU tests of the host-side logic around the kernels: the training view
schedule, the ADC schedule, hindsight relabelling of logged ADC decisions,
class weights, the Bezier-fit curve generator and the fit loop (against a
fake trainer)."""
import math

import numpy as np


def test_view_schedule_is_a_per_epoch_permutation():
    from nprush_b200.train import view_schedule
    for seed in (0, 7):
        seen = []
        for s in range(4):  # one epoch of 32 cameras, 8 per step
            v = view_schedule(s, 32, 8, seed)
            assert len(v) == 8 and np.all(np.diff(v) > 0)
            seen.append(v)
        np.testing.assert_array_equal(np.sort(np.concatenate(seen)), np.arange(32))
        np.testing.assert_array_equal(view_schedule(5, 32, 8, seed), view_schedule(5, 32, 8, seed))
    assert not np.array_equal(view_schedule(0, 32, 8, 0), view_schedule(4, 32, 8, 0))


def test_adc_schedule():
    from nprush_b200.train import AdcSchedule
    a = AdcSchedule()
    due = [s for s in range(1, 30001) if a.due(s)]
    assert due[0] == 500 and due[-1] == 15000 and len(due) == 146
    assert not AdcSchedule(every=0).due(500)


def test_hindsight_labels():
    from nprush_b200.learned_adc import AdcLog, class_weights, hindsight_labels
    log = AdcLog()
    # event 0: ids 1..5 with plain decisions keep, clone, split, prune, keep
    log.features = [np.zeros((5, 16), np.float32), np.zeros((2, 16), np.float32)]
    log.plain = [np.array([0, 1, 2, 3, 0], np.uint8), np.array([0, 0], np.uint8)]
    log.ids = [np.array([1, 2, 3, 4, 5]), np.array([1, 6])]
    # event 1 prunes lineages 1 and 2 (and 9, not logged)
    log.pruned_ids = [np.array([4]), np.array([1, 2, 9])]
    X, y = hindsight_labels(log, horizon=3)
    assert X.shape == (7, 16)
    # keep -> prune (1 pruned later); clone -> keep (2 pruned later); split, prune, keep unchanged
    np.testing.assert_array_equal(y[:5], [3, 0, 2, 3, 0])
    np.testing.assert_array_equal(y[5:], [0, 0])  # last event: no lookahead
    X0, y0 = hindsight_labels(log, horizon=0)
    np.testing.assert_array_equal(y0[:5], log.plain[0])
    w = class_weights(np.array([0] * 90 + [1] * 5 + [3] * 5, np.uint8))
    assert w[0] < 1.0 < w[1] and w[2] == 1.0 and math.isclose(w[1], w[3])  # absent class: weight 1


def test_random_walk_curves():
    from nprush_b200.bezier_fit import random_walk_curves
    b = random_walk_curves(4000, 5, height=512)
    assert b.shape == (4000, 20)
    assert np.all(np.abs(b[:, 0:3]) <= 1.0)
    steps = np.diff(b[:, [0, 4, 8, 12]], axis=1)
    assert 0.04 < steps.std() < 0.06
    px = b[:, 3] * 512 / 2
    assert px.min() >= 1.0 - 1e-5 and px.max() <= 3.0 + 1e-5
    assert np.all((b[:, 19] >= 0.3) & (b[:, 19] <= 1.0))


class _FakeTrainer:
    """Records the calls fit() makes (the kernels are not involved)."""

    def __init__(self):
        self.count = 100
        self.calls = []

    def set_graph(self, on):
        self.calls.append(("graph", bool(on)))

    def sync(self):
        pass

    def set_views(self, vp, vpi, sel):
        self.calls.append(("views", tuple(int(x) for x in sel)))

    def autotune(self):
        self.calls.append(("autotune",))
        return {"tile": 16, "fwd_form": 2, "per_tile": {}}

    def train_step(self, read_loss=False):
        self.calls.append(("step",))
        return (1.0, 0.0, 0.0) if read_loss else None

    def train_step_per_view(self, vp, vpi, sel, read_loss=False):
        self.calls.append(("step_per_view", tuple(int(x) for x in sel)))
        return None

    def adc(self, grad_thresh, split_scale, prune_opacity):
        self.calls.append(("adc",))
        self.count += 1
        return dict(before=self.count - 1, after=self.count, densified=1, pruned=0)

    def stats(self):
        return {"skipped_steps": 0}


def test_fit_autotunes_once_on_the_first_steps_views_and_times_adc():
    from nprush_b200.train import AdcSchedule, fit, view_schedule
    vp = np.zeros((32, 16), np.float32)
    t = _FakeTrainer()
    r = fit(t, vp, vp, 300, views=8, seed=3, adc=AdcSchedule(every=100, start=100, stop=200), mode="batched",
            autotune=True)
    names = [c[0] for c in t.calls]
    assert names.count("autotune") == 1 and r.tuned["tile"] == 16 and r.tune_s >= 0.0
    i = names.index("autotune")
    assert t.calls[i - 1] == ("views", tuple(int(x) for x in view_schedule(0, 32, 8, 3)))
    assert names.count("step") == 300 and names.count("adc") == 2
    assert [e[0] for e in r.adc_events] == [100, 200] and r.count == 102
    assert r.adc_s >= 0.0 and r.after_adc_s >= 0.0


def test_fit_per_view_mode_runs_eagerly_without_autotune():
    from nprush_b200.train import AdcSchedule, fit
    vp = np.zeros((16, 16), np.float32)
    t = _FakeTrainer()
    r = fit(t, vp, vp, 5, views=4, seed=0, adc=AdcSchedule(every=0), mode="per_view")
    names = [c[0] for c in t.calls]
    assert ("graph", False) in t.calls and "autotune" not in names and r.tuned is None
    assert names.count("step_per_view") == 5 and all(len(c[1]) == 4 for c in t.calls if c[0] == "step_per_view")
