"""Training driver for the Gaussian trainer (the fit-a-scene loop).

Schedule: each step trains on `views` cameras taken from a per-epoch
seeded permutation of all cameras; ADC (densify / prune) every `adc.every`
steps from `adc.start` up to `adc.stop`; PSNR over every camera at the end.

Two trainers share the kernels:
  * "batched": all views of a step in one launch per stage, the whole step
    replayed as one CUDA graph;
  * "per_view": the plain trainer, one eager launch sequence per view with
    the gradients accumulated, then one Adam update.

    python -m nprush_b200.train --steps 30000 --mode batched --out run.json
"""
from __future__ import annotations

import argparse
import functools
import json
import math
import time
from dataclasses import asdict, dataclass, field

import numpy as np


@dataclass
class AdcSchedule:
    every: int = 100
    start: int = 500
    stop: int = 15000
    grad_thresh: float = 2e-4
    split_scale: float = 0.01
    prune_opacity: float = 0.005

    def due(self, step: int) -> bool:
        """ADC runs after step `step` (1-based count of finished steps)."""
        return self.every > 0 and self.start <= step <= self.stop and step % self.every == 0


@dataclass
class FitResult:
    steps: int
    wall_s: float
    count: int
    adc_events: list = field(default_factory=list)
    losses: list = field(default_factory=list)
    psnr: list = field(default_factory=list)
    skipped_steps: int = 0
    adc_s: float = 0.0        # host time in the ADC calls (they end with the new count on the host)
    tune_s: float = 0.0       # host time of the raster autotuner
    tuned: dict | None = None
    after_adc_s: float = 0.0  # host time of the first step after each ADC event (batched: the re-capture)


@functools.lru_cache(maxsize=4)
def _epoch_perm(n_cams: int, seed: int, epoch: int) -> np.ndarray:
    return np.random.default_rng((seed, epoch)).permutation(n_cams)


def view_schedule(step: int, n_cams: int, views: int, seed: int) -> np.ndarray:
    """Cameras of step `step` (0-based): consecutive slices of a permutation
    drawn once per epoch from (seed, epoch)."""
    per_epoch = n_cams // views
    epoch, k = divmod(step, per_epoch)
    return np.sort(_epoch_perm(n_cams, seed, epoch)[k * views:(k + 1) * views])


def evaluate_psnr(trainer, vp, vpi, views: int = 8) -> np.ndarray:
    """Per-camera PSNR (dB) of the current parameters against the resident
    targets (target id = camera index)."""
    out = []
    n = vp.shape[0]
    for c0 in range(0, n, views):
        sel = np.arange(c0, min(c0 + views, n))
        trainer.set_views(vp[sel], vpi[sel], sel)
        trainer.forward()
        out.append(trainer.psnr())
    return np.concatenate(out)


def fit(trainer, vp, vpi, steps: int, views: int = 8, seed: int = 0, adc: AdcSchedule | None = None,
        mode: str = "batched", log_every: int = 0, adc_fn=None, autotune: bool = False) -> FitResult:
    """Train for `steps` steps; wall time covers training and ADC (and the
    autotuner when asked for), not the final evaluation.  adc_fn(trainer,
    step) replaces the plain ADC call when given (learned policies plug in
    here).  autotune: the raster autotuner chooses the tile size and raster
    variants on the first step's views before training."""
    n_cams = vp.shape[0]
    adc = adc or AdcSchedule()
    if mode == "batched":
        trainer.set_graph(True)
    elif mode == "per_view":
        trainer.set_graph(False)
    else:
        raise ValueError(mode)
    res = FitResult(steps=steps, wall_s=0.0, count=trainer.count)
    trainer.sync()
    t0 = time.perf_counter()
    if autotune and steps > 0:
        sel = view_schedule(0, n_cams, views, seed)
        trainer.set_views(vp[sel], vpi[sel], sel)
        res.tuned = trainer.autotune()
        res.tune_s = time.perf_counter() - t0
    after_adc = False
    for s in range(steps):
        sel = view_schedule(s, n_cams, views, seed)
        want_loss = log_every > 0 and (s % log_every == 0 or s == steps - 1)
        ts = time.perf_counter()
        if mode == "batched":
            trainer.set_views(vp[sel], vpi[sel], sel)
            l3 = trainer.train_step(read_loss=want_loss)
        else:
            l3 = trainer.train_step_per_view(vp[sel], vpi[sel], sel, read_loss=want_loss)
        if after_adc:
            res.after_adc_s += time.perf_counter() - ts
            after_adc = False
        if l3 is not None:
            res.losses.append((s + 1, l3[0]))
        if adc.due(s + 1):
            ta = time.perf_counter()
            if adc_fn is not None:
                ev = adc_fn(trainer, s + 1)
            else:
                ev = trainer.adc(adc.grad_thresh, adc.split_scale, adc.prune_opacity)
            res.adc_s += time.perf_counter() - ta
            after_adc = True
            res.adc_events.append((s + 1, ev["after"], ev["densified"], ev["pruned"]))
    trainer.sync()
    res.wall_s = time.perf_counter() - t0
    res.count = trainer.count
    res.skipped_steps = trainer.stats()["skipped_steps"]
    return res


def teacher_scene(device: int = 0, n_student: int = 200_000, n_teacher: int = 250_000, width: int = 800,
                  height: int = 800, n_cams: int = 32, sh_degree: int = 3, capacity: int | None = None,
                  student_seed: int = 10, teacher_seed: int = 11):
    """Seeded 200k / 800x800 training scene: cameras on a sphere, targets rendered on the GPU
    from a seeded teacher, a seeded student trainer with every target resident."""
    import torch

    from .gaussians import GaussianTrainer, orbit_cameras, random_gaussians
    vp, vpi = orbit_cameras(n_cams, width, height)
    teacher = GaussianTrainer(n_teacher, sh_degree=sh_degree, device=device,
                              params=random_gaussians(n_teacher, teacher_seed))
    tg = torch.zeros((n_cams, height, width, 4), device=f"cuda:{device}")
    teacher.set_image_size(width, height)
    for c0 in range(0, n_cams, 8):
        teacher.set_views(vp[c0:c0 + 8], vpi[c0:c0 + 8])
        teacher.forward(out=tg[c0:c0 + 8])
    teacher.close()
    tg[..., 3] = 1.0
    student = GaussianTrainer(capacity or n_student, sh_degree=sh_degree, device=device,
                              params=random_gaussians(n_student, student_seed))
    torch.cuda.synchronize()
    student.set_targets(tg, borrow=True)
    return vp, vpi, tg, student


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--mode", choices=("batched", "per_view"), default="batched")
    ap.add_argument("--gaussians", type=int, default=200_000)
    ap.add_argument("--teacher", type=int, default=250_000)
    ap.add_argument("--res", type=int, default=800)
    ap.add_argument("--width", type=int, default=None, help="image width (default: --res)")
    ap.add_argument("--height", type=int, default=None, help="image height (default: --res)")
    ap.add_argument("--cams", type=int, default=32, help="cameras on the sphere")
    ap.add_argument("--autotune", action="store_true", help="raster autotuner before training (batched)")
    ap.add_argument("--capacity", type=int, default=3_000_000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-adc", action="store_true")
    ap.add_argument("--adc-start", type=int, default=500)
    ap.add_argument("--adc-stop", type=int, default=15000)
    ap.add_argument("--log-every", type=int, default=1000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    import torch

    from . import _lib
    stream = torch.cuda.Stream(0)
    ctx = _lib.context(0)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    with torch.cuda.stream(stream):
        vp, vpi, tg, st = teacher_scene(0, a.gaussians, a.teacher, a.width or a.res, a.height or a.res,
                                        n_cams=a.cams, capacity=a.capacity)
        adc = AdcSchedule(every=0 if a.no_adc else 100, start=a.adc_start, stop=a.adc_stop)
        psnr0 = evaluate_psnr(st, vp, vpi)
        r = fit(st, vp, vpi, a.steps, seed=a.seed, adc=adc, mode=a.mode, log_every=a.log_every,
                autotune=a.autotune)
        r.psnr = evaluate_psnr(st, vp, vpi).tolist()
    out = dict(mode=a.mode, steps=a.steps, wall_s=r.wall_s, steps_per_s=a.steps / r.wall_s, count=r.count,
               psnr_mean=float(np.mean(r.psnr)), psnr_initial=float(np.mean(psnr0)), psnr=r.psnr,
               adc_events=r.adc_events, losses=r.losses, skipped_steps=r.skipped_steps, adc_s=r.adc_s,
               after_adc_s=r.after_adc_s, tune_s=r.tune_s, adc=asdict(adc), gaussians=a.gaussians,
               res=[a.width or a.res, a.height or a.res], cams=a.cams)
    line = json.dumps(out)
    print(json.dumps({k: out[k] for k in ("mode", "steps", "wall_s", "steps_per_s", "count", "psnr_mean",
                                          "psnr_initial", "skipped_steps", "adc_s", "after_adc_s", "tune_s")}))
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
