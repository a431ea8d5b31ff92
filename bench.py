"""Benchmark: train steps/s of the splat trainer on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--path compat]

Prints ONE JSON line (rank 0).  A step is one full training iteration over
the step's views (forward + loss + backward + Adam) on synthetic, seeded
inputs of the workload's shapes.  See DESIGN.md for the workload, the
algorithmic-byte model behind `roofline` and the CPU baseline.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------- workloads
def config2_cameras(n_cams=32, w=800, h=800, fov_deg=50.0, radius=4.0):
    from nprush_b200.camera import sphere_cameras
    return sphere_cameras(n_cams, radius, math.radians(fov_deg), w / h)


def compat_scene(n, seed):
    """Config-2 distribution in the reference's 16-float record: means U[-1,1]^3,
    scales exp(N(-4, 0.5)), random unit quaternions, opacity sigmoid(N(0,1)),
    RGB U[0,1], Gaussian shape (a=2, b=0.5)."""
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    sc = np.exp(rng.normal(-4.0, 0.5, (n, 3)))
    s[:, 3], s[:, 12], s[:, 15] = sc[:, 0], sc[:, 1], sc[:, 2]
    s[:, 4:7] = rng.random((n, 3))
    s[:, 7] = np.clip(1 / (1 + np.exp(-rng.normal(0, 1, n))), 0.06, 0.99)
    q = rng.normal(size=(n, 4))
    s[:, 8:12] = q / np.linalg.norm(q, axis=1, keepdims=True)
    s[:, 13], s[:, 14] = 2.0, 0.5
    return s


def run_compat(args, rank, world):
    """Reference-semantics trainer at the config-2 shape (200k splats, 800^2,
    8 of 32 views per step)."""
    import torch

    from nprush_b200 import _lib
    from nprush_b200.splat import GpuSplatOptimizerManager

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    n, w, h, vps = 200_000, 800, 800, 8
    vp, vpi = config2_cameras()
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    # teacher renders the targets for all 32 cameras
    teacher = GpuSplatOptimizerManager(250_000, device=dev, init=compat_scene(250_000, 11 + 1000 * rank))
    tg = torch.zeros((32, h, w, 4), device=f"cuda:{dev}")
    zero_t = torch.zeros((32, h, w, 4), device=f"cuda:{dev}")
    zero_d = torch.ones((32, h, w), device=f"cuda:{dev}")
    for c0 in range(0, 32, 8):
        teacher.write_splat_vp_matrix(vp[c0:c0 + 8], vpi[c0:c0 + 8])
        teacher.set_backward_target(zero_t[c0:c0 + 8], zero_d[c0:c0 + 8], w, h)
        teacher.backward(out_rgbd=tg[c0:c0 + 8])
    teacher.close()
    del zero_t, zero_d
    tgt_rgba = tg.clone()
    tgt_rgba[..., 3] = 1.0
    tgt_depth = tg[..., 3].contiguous()
    del tg
    student = GpuSplatOptimizerManager(n, device=dev, init=compat_scene(n, 10 + 1000 * rank))
    perm_rng = np.random.default_rng(1234 + rank)

    def views_for(step):
        perm = perm_rng.permutation(32)
        return np.sort(perm[:vps])

    flush = torch.empty(256 * 1024 * 1024 // 4, device=f"cuda:{dev}")

    def one_step(step):
        sel = views_for(step)
        student.write_splat_vp_matrix(vp[sel], vpi[sel])
        idx = torch.as_tensor(sel, device=f"cuda:{dev}")
        student.set_backward_target(tgt_rgba.index_select(0, idx), tgt_depth.index_select(0, idx), w, h)
        student.dispatch()

    with torch.cuda.stream(stream):
        for s in range(args.warmup):
            one_step(s)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        times = []
        with ClockSampler(dev) as clk:
            for s in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                one_step(args.warmup + s)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    ms = float(np.sum(times))
    st = student.stats()
    return dict(ms_total=ms, times=times, clocks=clk.summary(), pairs=st["pairs"], n=n, w=w, h=h, views=vps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="compat", choices=["compat"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "CPU reference leg not wired yet"}))
        return
    res = run_compat(args, rank, world)
    ms = res["ms_total"]
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * 1000.0 / ms_per_step
    if rank == 0:
        line = {
            "metric": "train steps/s (fwd+bwd+Adam, 200k splats, 800^2, 8 views)",
            "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded, teacher-rendered targets)",
            "config": {"workload": "reference-semantics splat trainer at the config-2 shape", "splats": res["n"],
                       "resolution": [res["w"], res["h"]], "views_per_step": res["views"],
                       "l2": "flushed between steps", "pairs_last_step": res["pairs"]},
            "clocks": res["clocks"],
        }
        print(json.dumps(line))


if __name__ == "__main__":
    main()
