"""Hindsight labelling of the learned ADC (CPU): the plain rule's logged
decisions are relabelled by what the plain rule later did to each lineage."""
import numpy as np

from nprush_b200.learned_adc import AdcLog, hindsight_labels, per_class_recall


def _log(events):
    """events: list of (ids, plain decisions, split preference) per ADC event."""
    log = AdcLog()
    for ids, plain, pref in events:
        ids = np.asarray(ids, np.int32)
        plain = np.asarray(plain, np.uint8)
        log.features.append(np.zeros((len(ids), 16), np.float32) + np.arange(len(ids))[:, None])
        log.plain.append(plain)
        log.ids.append(ids)
        log.pruned_ids.append(np.unique(ids[plain == 3]))
        log.densified_ids.append(np.unique(ids[(plain == 1) | (plain == 2)]))
        log.split_pref.append(np.asarray(pref, np.uint8))
    return log


def test_relabelling_rules():
    # event 0: ids 0..5; event 1: lineage 1 pruned, lineage 2 split, lineage 3 cloned,
    # lineage 5 densified and later pruned (event 2)
    log = _log([
        ([0, 1, 2, 3, 4, 5], [0, 0, 0, 0, 2, 0], [2, 2, 2, 1, 2, 2]),
        ([0, 1, 2, 3, 4, 5], [0, 3, 2, 1, 0, 2], [2, 2, 2, 1, 2, 2]),
        ([0, 2, 3, 4, 5], [0, 0, 0, 0, 3], [2, 2, 1, 2, 2]),
    ])
    X, y = hindsight_labels(log, horizon=3)
    first = y[:6]
    assert first[0] == 0          # nothing happens to lineage 0: keep
    assert first[1] == 3          # pruned later: prune now
    assert first[2] == 2          # split at the next event, never pruned: split now
    assert first[3] == 1          # cloned at the next event (small scale): clone now
    assert first[4] == 2          # the plain rule split it and the lineage survives: stays split
    assert first[5] == 3          # densified next, but pruned within the horizon: prune now
    # without the densify-earlier rule only the prune relabelling applies
    _, y2 = hindsight_labels(log, horizon=3, densify_early=False)
    assert list(y2[:6]) == [0, 3, 0, 0, 2, 3]
    # a densification whose lineage is pruned later becomes keep
    assert y[6 + 5] == 0
    assert X.shape == (6 + 6 + 5, 16)


def test_per_class_recall():
    conf = np.array([[8, 1, 0, 1], [0, 0, 0, 0], [1, 0, 3, 0], [2, 0, 0, 2]])
    r = per_class_recall(conf)
    assert r[0] == 0.8 and r[1] is None and r[2] == 0.75 and r[3] == 0.5
