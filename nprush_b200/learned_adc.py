"""Learned ADC: logging plain-ADC decisions, hindsight labels, training the
policy network, and running ADC with it.

Labels come from the plain threshold rule's own runs.  At every ADC event the
16-float features of a sample of Gaussians are logged with the plain decision
and each Gaussian's lineage id (inherited by clones and split children).  A
logged decision is then relabelled by what happened to the lineage over the
next `horizon` events:

  * keep  -> prune  when the plain rule prunes a member of the lineage later
    (the Gaussian was dead weight: prune it now);
  * keep  -> clone / split (by the Gaussian's own largest scale, as the plain
    rule chooses) when the plain rule densifies the lineage at the next event
    and prunes none of it within the horizon (it was going to be densified:
    do it one event earlier);
  * clone / split -> keep  when a member of the lineage is pruned later (the
    densification did not pay);
  * prune stays prune.

The network therefore learns the plain rule plus earlier pruning and fewer
wasted densifications.  The plain rule stays the fallback (no network, or a
Gaussian whose logits are not finite) and the judge: the A/B run compares
final PSNR, Gaussian count and wall time against it.

    python -m nprush_b200.learned_adc --log-seeds 100 101 --eval-seeds 120 121 122 --steps 3000 --out ab.json
"""
from __future__ import annotations

import argparse
import json
from dataclasses import dataclass, field

import numpy as np

from .train import AdcSchedule, evaluate_psnr, fit


@dataclass
class AdcLog:
    samples_per_event: int = 20000
    seed: int = 0
    features: list = field(default_factory=list)   # per event [k, 16]
    plain: list = field(default_factory=list)      # per event [k]
    ids: list = field(default_factory=list)        # per event [k]
    pruned_ids: list = field(default_factory=list)  # per event: sorted ids the plain rule pruned
    densified_ids: list = field(default_factory=list)  # per event: sorted ids the plain rule cloned or split
    split_pref: list = field(default_factory=list)  # per event [k]: 2 if the Gaussian's largest scale calls for a split

    def record(self, trainer, step_frac: float, adc: AdcSchedule):
        feat, plain, ids = trainer.adc_features(step_frac, adc.grad_thresh, adc.split_scale, adc.prune_opacity)
        plain_h = plain.cpu().numpy()
        ids_h = ids.cpu().numpy()
        n = len(plain_h)
        rng = np.random.default_rng((self.seed, len(self.features)))
        k = min(self.samples_per_event, n)
        sel = np.sort(rng.choice(n, k, replace=False)) if k < n else np.arange(n)
        self.features.append(feat.cpu().numpy()[sel])
        self.plain.append(plain_h[sel])
        self.ids.append(ids_h[sel])
        self.pruned_ids.append(np.unique(ids_h[plain_h == 3]))
        self.densified_ids.append(np.unique(ids_h[(plain_h == 1) | (plain_h == 2)]))
        # feature 7 is (largest log-scale - log split_scale) / ln 10: > 0 means split
        self.split_pref.append(np.where(feat.cpu().numpy()[sel][:, 7] > 0, 2, 1).astype(np.uint8))


def hindsight_labels(log: AdcLog, horizon: int = 3, densify_early: bool = True):
    """(features [N,16], labels [N]) relabelled by the lineages' fate."""
    X, Y = [], []
    ev = len(log.features)
    for e in range(ev):
        y = log.plain[e].astype(np.uint8).copy()
        later = [log.pruned_ids[j] for j in range(e + 1, min(ev, e + 1 + horizon))]
        dead = np.isin(log.ids[e], np.unique(np.concatenate(later))) if later else np.zeros(len(y), bool)
        if densify_early and e + 1 < ev and log.densified_ids:
            soon = np.isin(log.ids[e], log.densified_ids[e + 1]) & ~dead
            keep = y == 0
            y[keep & soon] = log.split_pref[e][keep & soon]
        y[(y == 0) & dead] = 3
        y[((y == 1) | (y == 2)) & dead] = 0
        X.append(log.features[e])
        Y.append(y)
    return np.concatenate(X), np.concatenate(Y)


def per_class_recall(conf: np.ndarray) -> list:
    """Recall of each class (keep, clone, split, prune) from a confusion
    matrix [true, predicted]; None for a class with no samples."""
    tot = conf.sum(axis=1)
    return [None if tot[k] == 0 else float(conf[k, k] / tot[k]) for k in range(conf.shape[0])]


def class_weights(y, cap: float = 20.0):
    cnt = np.bincount(y, minlength=4).astype(np.float64)
    w = np.where(cnt > 0, cnt.sum() / (4.0 * np.maximum(cnt, 1.0)), 1.0)
    return np.clip(w, 1.0 / cap, cap).astype(np.float32)


def logging_adc_fn(log: AdcLog, adc: AdcSchedule):
    def fn(trainer, step):
        log.record(trainer, step / adc.stop, adc)
        return trainer.adc(adc.grad_thresh, adc.split_scale, adc.prune_opacity)
    return fn


def plain_adc_fn(adc: AdcSchedule):
    def fn(trainer, step):
        return trainer.adc(adc.grad_thresh, adc.split_scale, adc.prune_opacity)
    return fn


def policy_adc_fn(policy, adc: AdcSchedule, margin: float = 0.0):
    def fn(trainer, step):
        trainer.set_policy_margin(margin)
        return trainer.adc_policy(policy, step / adc.stop, adc.grad_thresh, adc.split_scale, adc.prune_opacity)
    return fn


def run(scene_fn, steps: int, seed: int, adc: AdcSchedule, adc_fn=None, mode: str = "batched", views: int = 8,
        autotune: bool = False):
    """One training run on a fresh scene; returns (FitResult, mean PSNR)."""
    vp, vpi, tg, st = scene_fn(seed)
    st.assign_ids(0)
    r = fit(st, vp, vpi, steps, views=views, seed=seed, adc=adc, mode=mode, adc_fn=adc_fn, autotune=autotune)
    psnr = float(np.mean(evaluate_psnr(st, vp, vpi, views=views)))
    st.close()
    return r, psnr


def _tile_choice(tuned):
    """The autotuner's choice without its timing table."""
    return None if tuned is None else {k: v for k, v in tuned.items() if k != "per_tile"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--log-seeds", type=int, nargs="+", default=[100, 101])
    ap.add_argument("--eval-seeds", type=int, nargs="+", default=[120],
                    help="held-out scenes: every arm trains each of them")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--log-steps", type=int, default=None,
                    help="length of the logging runs (default: up to the last ADC event)")
    ap.add_argument("--margins", type=float, nargs="+", default=[0.0],
                    help="keep-logit margins of the learned arms (one evaluation run each)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain batched arm")
    ap.add_argument("--with-per-view", action="store_true",
                    help="also run the plain per-view trainer (eager, one view per launch, default raster "
                         "variants) on the eval seed")
    ap.add_argument("--with-per-view-tuned", action="store_true",
                    help="also run the per-view trainer with the autotuned raster variants (context)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batched arms keep the default raster variants (the autotuner is part of the batched "
                         "trainer and its time counts in their wall time)")
    ap.add_argument("--adc-stop", type=int, default=None)
    ap.add_argument("--adc-start", type=int, default=500)
    ap.add_argument("--adc-every", type=int, default=100)
    ap.add_argument("--sh-degree", type=int, default=3)
    ap.add_argument("--deterministic", action="store_true", help="bit-reproducible training runs")
    ap.add_argument("--plain-thresholds", type=float, nargs="*", default=[],
                    help="extra plain arms with these densification thresholds (the count / PSNR trade-off "
                         "the plain rule itself offers)")
    ap.add_argument("--gaussians", type=int, default=200_000)
    ap.add_argument("--teacher", type=int, default=250_000)
    ap.add_argument("--res", type=int, default=800)
    ap.add_argument("--width", type=int, default=None, help="image width (default: --res)")
    ap.add_argument("--height", type=int, default=None, help="image height (default: --res)")
    ap.add_argument("--horizon", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--no-densify-early", action="store_true",
                    help="leave out the keep -> densify relabelling (densified at the next event anyway)")
    ap.add_argument("--views", type=int, default=8, help="views per step")
    ap.add_argument("--cams", type=int, default=32, help="cameras on the sphere")
    ap.add_argument("--log-gaussians", type=int, default=None,
                    help="scene of the logging runs (default: the evaluation scene's); e.g. the 200k / 800x800 / "
                         "32-camera scene for a policy evaluated at 1M / 1920x1080 / 64 cameras")
    ap.add_argument("--log-teacher", type=int, default=None)
    ap.add_argument("--log-res", type=int, default=None)
    ap.add_argument("--log-cams", type=int, default=None)
    ap.add_argument("--class-weights", action="store_true",
                    help="weight classes by inverse frequency (default: uniform; a false prune costs more "
                         "than a missed one)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    import torch

    from . import _lib
    from .policy import AdcPolicy
    from .train import teacher_scene
    stream = torch.cuda.Stream(0)
    ctx = _lib.context(0)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    adc = AdcSchedule(every=a.adc_every, start=a.adc_start, stop=a.adc_stop or min(15000, a.steps))

    def make_scene(gaussians, teacher, width, height, cams):
        def scene(seed):
            # student and teacher seeds derived from the run seed
            vp, vpi, tg, st = teacher_scene(0, gaussians, teacher, width, height, n_cams=cams,
                                            sh_degree=a.sh_degree, capacity=4 * gaussians, student_seed=seed,
                                            teacher_seed=seed + 1000)
            if a.deterministic:
                st.set_deterministic(True)
            return vp, vpi, tg, st
        return scene

    scene = make_scene(a.gaussians, a.teacher, a.width or a.res, a.height or a.res, a.cams)
    log_scene = scene
    if a.log_gaussians or a.log_res or a.log_cams or a.log_teacher:
        lg = a.log_gaussians or a.gaussians
        log_scene = make_scene(lg, a.log_teacher or a.teacher, a.log_res or a.width or a.res,
                               a.log_res or a.height or a.res, a.log_cams or a.cams)

    out = {}
    with torch.cuda.stream(stream):
        log = AdcLog(seed=1)
        log_steps = a.log_steps or min(a.steps, adc.stop)
        for s in a.log_seeds:
            r, p = run(log_scene, log_steps, s, adc, logging_adc_fn(log, adc))
            out.setdefault("log_runs", []).append(dict(seed=s, psnr=p, count=r.count, wall_s=r.wall_s))
        X, y = hindsight_labels(log, a.horizon, densify_early=not a.no_densify_early)
        cw = class_weights(y) if a.class_weights else np.ones(4, np.float32)
        # hold out every 10th sample to score the network
        hold = np.arange(len(y)) % 10 == 0
        pol = AdcPolicy(seed=7)
        lc, ac = pol.train(X[~hold], y[~hold], epochs=a.epochs, batch=8192, lr=2e-3, seed=3, class_w=cw)
        z = pol.logits(X[hold]).cpu().numpy()
        pred = np.argmax(np.c_[np.zeros(len(z)), z], axis=1)
        conf = np.zeros((4, 4), np.int64)
        np.add.at(conf, (y[hold], pred), 1)
        out["training"] = dict(samples=int(len(y)), class_counts=np.bincount(y, minlength=4).tolist(),
                               class_w=cw.tolist(), loss=lc.tolist(), acc=ac.tolist(),
                               heldout_confusion=conf.tolist(), heldout_recall=per_class_recall(conf))
        tune = not a.no_autotune
        arms = [] if a.no_plain else [("plain", None, "batched", tune)]
        for thr in a.plain_thresholds:
            arms.append((f"plain_t{thr:g}", plain_adc_fn(AdcSchedule(every=adc.every, start=adc.start,
                                                                     stop=adc.stop, grad_thresh=thr)), "batched",
                         tune))
        for mg in a.margins:
            arms.append(("learned" if mg == 0.0 else f"learned_m{mg:g}", policy_adc_fn(pol, adc, mg), "batched",
                         tune))
        if a.with_per_view:
            arms.append(("plain_per_view", None, "per_view", False))
        if a.with_per_view_tuned:
            arms.append(("plain_per_view_tuned", None, "per_view", True))
        for name, fn, mode, at in arms:
            runs = []
            for es in a.eval_seeds:
                r, p = run(scene, a.steps, es, adc, fn, mode=mode, views=a.views, autotune=at)
                runs.append(dict(seed=es, psnr=p, count=r.count, wall_s=r.wall_s, steps_per_s=a.steps / r.wall_s,
                                 adc_s=r.adc_s, after_adc_s=r.after_adc_s, tune_s=r.tune_s, tuned=_tile_choice(r.tuned),
                                 skipped=r.skipped_steps, adc_events=r.adc_events[-3:]))
            out[name] = dict(mode=mode, runs=runs, psnr=float(np.mean([x["psnr"] for x in runs])),
                             count=float(np.mean([x["count"] for x in runs])),
                             wall_s=float(np.mean([x["wall_s"] for x in runs])))
        if "plain" in out:
            for name in [k for k in out if k.startswith("learned") or k.startswith("plain_t")]:
                d_psnr = [x["psnr"] - y["psnr"] for x, y in zip(out[name]["runs"], out["plain"]["runs"])]
                d_cnt = [x["count"] / y["count"] - 1.0 for x, y in zip(out[name]["runs"], out["plain"]["runs"])]
                out[name]["vs_plain"] = dict(psnr_db=d_psnr, count_frac=d_cnt)
        if "plain_per_view" in out:
            # the target's comparison: batched arms against the plain per-view trainer
            base = out["plain_per_view"]
            for name in [k for k in out if k in ("plain", "plain_per_view_tuned") or k.startswith("learned")]:
                out[name]["vs_per_view"] = dict(wall_frac=out[name]["wall_s"] / base["wall_s"],
                                                psnr_db=out[name]["psnr"] - base["psnr"])
    out["config"] = vars(a)
    print(json.dumps({k: v for k, v in out.items() if k not in ("training", "log_runs", "config")}))
    print(json.dumps(dict(class_counts=out["training"]["class_counts"], acc=out["training"]["acc"][-1],
                          confusion=out["training"]["heldout_confusion"],
                          recall=out["training"]["heldout_recall"])))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f)


if __name__ == "__main__":
    main()
