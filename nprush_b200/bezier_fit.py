"""Cubic 3D Bezier curve fitting (50k curves, 512x512, 4 views per step), through the
reference-semantics Bezier optimiser (GpuBezierOptimizerManager).

Scene: curves built as random walks (start U[-1,1]^3, steps N(0, 0.05)),
widths 1-3 px log-uniform converted to NDC units (2 px / H), RGB U[0,1],
opacity U[0.3, 1]; a seeded 60k-curve teacher rendered by the headless
display forward gives the 512 x 512 targets of 32 sphere cameras (r = 4,
fov 50 deg); the 50k-curve student fits 4 views per dispatch (backward over
the 4 views, Adam step, ADC every adc_period dispatches), each curve drawn
as a 16-segment screen-space ribbon.

    python -m nprush_b200.bezier_fit --steps 200 --out fit.json
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np


def random_walk_curves(n: int, seed: int, height: int = 512) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 20), np.float32)
    p = rng.uniform(-1, 1, (n, 3))
    for k in range(4):
        if k:
            p = p + rng.normal(0, 0.05, (n, 3))
        b[:, 4 * k:4 * k + 3] = p
    px = np.exp(rng.uniform(math.log(1.0), math.log(3.0), n))
    b[:, 3] = 2.0 * px / height      # width, NDC units
    b[:, 7] = 0.5 * b[:, 3]          # edge softness
    b[:, 16:19] = rng.random((n, 3))
    b[:, 19] = rng.uniform(0.3, 1.0, n)
    return b


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--curves", type=int, default=50_000)
    ap.add_argument("--teacher", type=int, default=60_000)
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--views", type=int, default=4)
    ap.add_argument("--cams", type=int, default=32)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--adc-period", type=int, default=50)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    import torch

    from . import _lib
    from .bezier import GpuBezierOptimizerManager
    from .camera import sphere_cameras
    dev = 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    W = H = a.res
    vp, vpi = sphere_cameras(a.cams, 4.0, math.radians(50.0), 1.0)
    with torch.cuda.stream(stream):
        teacher = GpuBezierOptimizerManager(a.teacher, init=random_walk_curves(a.teacher, 21, H))
        tg = torch.zeros((a.cams, H, W, 4), device="cuda")
        for c in range(a.cams):
            teacher.render(vp[c], W, H, tg[c])
        teacher.close()
        student = GpuBezierOptimizerManager(a.curves, init=random_walk_curves(a.curves, 20, H))
        student.write_mode(1.0)
        student.set_adc_period(a.adc_period)
        depth = torch.ones((a.views, H, W, 4), device="cuda")
        zeros = torch.zeros((a.views, H, W, 4), device="cuda")
        rng = np.random.default_rng(5)

        def step(k):
            sel = np.sort(rng.permutation(a.cams)[:a.views])
            student.write_vp(vp[sel], vpi[sel])
            student.set_backward_target(tg[torch.as_tensor(sel, device="cuda")].contiguous(), depth, zeros, depth,
                                        zeros, W, H)
            student.dispatch()

        def psnr():
            out = torch.zeros((H, W, 4), device="cuda")
            vals = []
            for c in range(0, a.cams, 4):
                student.render(vp[c], W, H, out)
                mse = torch.mean((out[..., :3] - tg[c, ..., :3]) ** 2).item()
                vals.append(-10 * math.log10(max(mse, 1e-12)))
            return float(np.mean(vals))

        p0 = psnr()
        for k in range(a.warmup):
            step(k)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for k in range(a.steps):
            step(a.warmup + k)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        wall = (time.perf_counter() - t0) / a.steps * 1000.0
        st = student.stats()
        p1 = psnr()
    res = dict(workload=f"{a.curves // 1000}k cubic Bezier curves, {W}x{H}, {a.views} of {a.cams} "
                        "cameras per dispatch, 16-segment ribbons, reference semantics",
               steps_per_s=1000.0 / ms, ms_per_step=ms, host_ms_per_step=wall, steps=a.steps,
               pairs=st["pairs"], psnr_before=p0, psnr_after=p1)
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)


if __name__ == "__main__":
    main()
