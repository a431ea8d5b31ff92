"""Benchmark: train steps/s (fwd + bwd + Adam, 200k Gaussians SH3, 800x800,
8 views per step) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

Prints ONE JSON line (rank 0).  A step is one full training iteration over 8
of 32 sphere cameras (forward + L1/D-SSIM loss + backward + Adam) on seeded
synthetic inputs: a 200k-Gaussian student fitted to images rendered from a
250k-Gaussian teacher.  `value` is timed with CUDA events on the library's
stream with everything resident in HBM; `e2e` goes through the public API with
the step's 8 target images uploaded from page-locked host memory every step
(the next step's upload overlapping the current step) and the loss read back
every step.  `--impl reference` times the reference's own shader code
for this path (translated to C++, oracle/_ref) on the host, on a bounded
sample of the same shape.  With N > 1 GPUs each step's 8 views are split
over the ranks (view-sharded data parallelism: one NCCL all-reduce of the
gradients per step, Adam on every replica; strong scaling).
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

N_GAUSS, N_TEACHER, WIDTH, HEIGHT, VIEWS, CAMS, SH_DEG = 200_000, 250_000, 800, 800, 8, 32, 3  # 200k Gaussians SH3, 800x800, 8 of 32 views
P_USED = 59          # floats per Gaussian used by the model
# DRAM traffic of one backward-raster launch (dram__bytes_read.sum + dram__bytes_write.sum) from one
# 1-pass ncu capture of this workload (11,433,806 pairs): scaled to a launch by its pair count.
BWD_TRAFFIC_BYTES, BWD_TRAFFIC_PAIRS = 239_281_152 + 18_662_144, 11_433_806
S_REC = 36           # algorithmic projected-record bytes (mean2d, conic, rgb, opacity)
# Warp instructions issued by one launch of each raster kernel (smsp__inst_executed.sum) in a 1-pass
# ncu capture of this workload with the variant named, and that launch's pair count: scaled to a
# launch by its pair count.  Key: (stage, form, pixels per thread, records per stage) at 16 x 16 tiles.
RASTER_INST = {("raster_fwd", 2, 2, 128): (548_836_695, 11_433_806),
               ("raster_bwd", 2, 2, 128): (1_183_662_764, 11_433_806)}
SMS, ISSUE_PER_SM_CLK = 148, 4  # B200: 148 SMs, four warp schedulers each issuing one instruction per clock


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
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


def stage_bytes(stage: str, V: int, N: int, K: int, npx: int, tile_passes: int) -> float:
    """Algorithmic (compulsory) bytes of one launch of a stage of the step."""
    return {
        "preprocess": V * N * (P_USED * 4 + S_REC + 20),
        "depth_sort": 4 * 16 * V * N,
        "emit": V * N * 16 + K * 8,
        "tile_sort": tile_passes * 16 * K,
        "ranges": K * 4 + 8 * V * npx / 256,
        "raster_fwd": K * (4 + S_REC) + V * npx * (12 + 8),
        "loss": V * npx * (12 + 12 + 12),
        "raster_bwd": K * (4 + S_REC) + V * npx * (12 + 8 + 12) + V * N * 40,
        "project_bwd": V * N * (40 + S_REC) + 2 * N * P_USED * 4,
        "adam": N * P_USED * 4 * 7,
    }[stage]


def issue_roofline(stage, tuned, K, ms, sm_mhz):
    """Issue-slot roofline of a raster stage: its warp instructions per launch (the ncu count of the same
    variant, scaled by pairs) over its CUDA-event duration, against SMs x 4 schedulers x the SM clock
    sampled during the timed steps.  None when no count of the variant that ran is recorded."""
    if tuned is None or tuned["tile"] != 16:
        return None
    form, ppt, sps = ((tuned["fwd_form"], tuned["fwd_ppt"], tuned["fwd_stage"]) if stage == "raster_fwd" else
                      (tuned["bwd_form"], tuned["bwd_ppt"], tuned["bwd_stage"]))
    rec = RASTER_INST.get((stage, form, ppt, sps))
    if rec is None or not ms:
        return None
    inst = rec[0] * K / rec[1]
    mhz = sm_mhz or 1965.0
    achieved = inst / (ms * 1e-3) / 1e9
    peak = SMS * ISSUE_PER_SM_CLK * mhz * 1e-3
    return {"bound": "issue", "kernel": stage, "achieved": achieved, "peak": peak, "unit": "G warp-inst/s",
            "frac": achieved / peak, "inst_per_launch": inst, "sm_mhz": mhz,
            "source": "ncu smsp__inst_executed.sum of the same variant at this workload, scaled by pairs"}


def step_bytes(V, N, K, npx):
    """Whole-step compulsory bytes (forward + backward + Adam)."""
    fwd = V * N * P_USED * 4 + V * N * S_REC + K * 8 + K * (8 + S_REC) + V * npx * 12
    bwd = K * (8 + S_REC) + V * npx * (12 + 8) + V * N * S_REC + V * N * (S_REC + P_USED * 4) + N * P_USED * 4
    return fwd + bwd + N * P_USED * 4 * 7


# ----------------------------------------------------------------- our arm
def build_scene(dev):
    import torch

    from nprush_b200.gaussians import GaussianTrainer, orbit_cameras, random_gaussians
    vp, vpi = orbit_cameras(CAMS, WIDTH, HEIGHT)
    teacher = GaussianTrainer(N_TEACHER, sh_degree=SH_DEG, device=dev, params=random_gaussians(N_TEACHER, 11))
    tg = torch.zeros((CAMS, HEIGHT, WIDTH, 4), device=f"cuda:{dev}")
    teacher.set_image_size(WIDTH, HEIGHT)
    for c0 in range(0, CAMS, VIEWS):
        teacher.set_views(vp[c0:c0 + VIEWS], vpi[c0:c0 + VIEWS])
        teacher.forward(out=tg[c0:c0 + VIEWS])
    teacher.close()
    tg[..., 3] = 1.0
    student = GaussianTrainer(N_GAUSS, sh_degree=SH_DEG, device=dev, params=random_gaussians(N_GAUSS, 10))
    return vp, vpi, tg, student


def view_schedule(steps: int):
    """The cameras of each step: VIEWS of the CAMS sphere cameras, drawn by a
    seeded permutation per step, in ascending order."""
    rng = np.random.default_rng(1234)
    return [np.sort(rng.permutation(CAMS)[:VIEWS]) for _ in range(steps)]


def run_ours(args, rank, world):
    import torch

    from nprush_b200 import _lib
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    with torch.cuda.stream(stream):
        vp, vpi, tg, st = build_scene(dev)
        torch.cuda.synchronize()
        st.set_targets(tg, borrow=True)
        sched = view_schedule(args.warmup + args.steps + 4)
        tuned = fixed = None
        if args.raster:
            # a fixed tile and raster variants: tile,fwd form,ppt,stage,bwd form,ppt,stage
            r7 = [int(x) for x in args.raster.split(",")]
            st.set_tile(r7[0])
            st.set_raster(r7[1:4], r7[4:7])
            fixed = dict(zip(("tile", "fwd_form", "fwd_ppt", "fwd_stage", "bwd_form", "bwd_ppt", "bwd_stage"), r7))
        elif not args.no_autotune:
            # tile size and raster variants timed on this workload
            st.set_views(vp[sched[0]], vpi[sched[0]], sched[0])
            tuned = st.autotune()
        st.set_graph(not args.no_graph)  # whole step captured as one CUDA graph
        # stage timers are event-record nodes of the graph, so they must be on
        # when the first (capturing) step runs
        st.set_timing(not args.no_stage_timing)
        flush = torch.empty(64 * 1024 * 1024, device=f"cuda:{dev}")  # 256 MB > L2

        def step(k):
            sel = sched[k]
            st.set_views(vp[sel], vpi[sel], sel)
            st.train_step()

        for k in range(args.warmup):
            step(k)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        st.stage_times(reset=True)
        times, pairs = [], []
        torch.cuda.nvtx.range_push("timed_steps")  # lets a profiler take the timed steps' launches alone
        with ClockSampler(dev) as clk:
            for k in range(args.steps):
                if not args.no_flush:
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step(args.warmup + k)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                pairs.append(st.stats()["pairs"])
        torch.cuda.nvtx.range_pop()
        stages = st.stage_times(reset=True)
        # kernels launched per step: the captured step's kernel nodes (graph mode)
        graph_kernels = st.stats()["graph_kernels"] if not args.no_graph else None
        st.set_timing(False)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        # ---- end to end through the public API with host buffers: every step
        # uploads its 8 target images from page-locked host memory (the next
        # step's upload runs on a side stream while the current step computes)
        # and reads its loss back
        host_all = torch.empty((CAMS, HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True)
        host_all.copy_(tg.cpu())
        hs = host_all.numpy()
        local = np.arange(VIEWS, dtype=np.uint32)

        def e2e_step(k, prefetch):
            sel = sched[k]
            st.set_views(vp[sel], vpi[sel], local)
            st.train_step()
            if prefetch:
                st.upload_targets(hs, sched[k + 1])  # H2D of the next step's inputs
            return st.read_loss()                    # D2H of this step's result

        st.upload_targets(hs, sched[0])
        e2e_step(0, True)  # the first step on the uploaded targets re-captures the graph: untimed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(1, args.steps + 1):
            loss_last = e2e_step(k, k < args.steps)
        e2e_times = [(time.perf_counter() - t0) * 1000.0 / args.steps]
        h2d = VIEWS * HEIGHT * WIDTH * 4 * 4 + VIEWS * (32 * 4 + 4)
        d2h = 3 * 4
        st.close()
        trained = (trained_state_leg(args, dev, stream, vp, vpi, tg, tuned if tuned is not None else fixed, flush,
                                     retune=tuned is not None) if args.trained_steps > 0 else None)
    return dict(tuned=tuned, ms_total=float(np.sum(times)), times=times, stages=stages, pairs=int(np.mean(pairs)),
                trained=trained,
                graph_kernels=graph_kernels,
                clocks=clk.summary(), e2e_ms=float(np.mean(e2e_times)), h2d=h2d, d2h=d2h, loss=loss_last)


def run_sharded(args, rank, world):
    """N > 1: the view-sharded trainer (nprush_b200.distributed): each rank
    renders its share of a step's 8 views on a full replica of the 200k
    Gaussians, one NCCL all-reduce of the gradient buffer per step, Adam on
    every replica (strong scaling: the step's work is fixed, split over the
    ranks).  Timed like the single-GPU line: CUDA events around each step,
    L2 flushed between steps, the max over ranks taken by the caller."""
    import torch

    from nprush_b200 import _lib
    from nprush_b200.distributed import ShardedTrainer, shard_views
    from nprush_b200.gaussians import random_gaussians
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    mine = shard_views(VIEWS, rank, world)
    with torch.cuda.stream(stream):
        vp, vpi, tg, st = build_scene(dev)
        torch.cuda.synchronize()
        st.set_targets(tg, borrow=True)
        sched = view_schedule(args.warmup + args.steps + 4)
        tuned = None
        sel0 = sched[0][mine]
        if not args.no_autotune and len(mine):
            st.set_views(vp[sel0], vpi[sel0], sel0)
            tuned = st.autotune()
        # kernels of this rank's step: its graph captured once (the sharded
        # step launches the same kernels eagerly), then eager steps
        graph_kernels = 0
        if len(mine):
            st.set_graph(True)
            st.set_views(vp[sel0], vpi[sel0], sel0)
            st.train_step()
            st.train_step()
            graph_kernels = st.stats()["graph_kernels"]
            st.set_graph(False)
            # back to the common starting point (those two steps saw only this rank's views)
            zeros = np.zeros((N_GAUSS, 64), np.float32)
            st.write_params(random_gaussians(N_GAUSS, 10))
            st.write_state(zeros, zeros, 0)
            st.write_adc_stats(np.zeros(N_GAUSS, np.float32), np.zeros(N_GAUSS, np.float32))
        sh = ShardedTrainer(st)
        st.set_timing(True)
        flush = torch.empty(64 * 1024 * 1024, device=f"cuda:{dev}")
        for k in range(args.warmup):
            sh.train_step(vp[sched[k]], vpi[sched[k]], sched[k])
        torch.cuda.synchronize()
        torch.distributed.barrier()
        st.stage_times(reset=True)
        times, pairs = [], []
        with ClockSampler(dev) as clk:
            for k in range(args.steps):
                sel = sched[args.warmup + k]
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sh.train_step(vp[sel], vpi[sel], sel)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                pairs.append(st.stats()["pairs"])
        stages = st.stage_times(reset=True)
        st.set_timing(False)
        torch.cuda.synchronize()
        torch.distributed.barrier()
        # end to end: each rank uploads its own views' targets from page-locked host memory and reads its
        # share of the loss back every step
        host_all = torch.empty((CAMS, HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True)
        host_all.copy_(tg.cpu())
        hs = host_all.numpy()
        ids = np.zeros(VIEWS, np.uint32)
        ids[mine] = np.arange(len(mine), dtype=np.uint32)
        torch.distributed.barrier()
        t0 = time.perf_counter()
        for k in range(args.steps):
            sel = sched[k]
            if len(mine):
                st.upload_targets(hs, sel[mine])
            loss_last = sh.train_step(vp[sel], vpi[sel], ids)
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        st.close()
    return dict(tuned=tuned, ms_total=float(np.sum(times)), times=times, stages=stages, pairs=int(np.mean(pairs)),
                trained=None, graph_kernels=graph_kernels * world, views_local=len(mine), scaling="strong",
                clocks=clk.summary(), e2e_ms=e2e_ms, h2d=len(mine) * HEIGHT * WIDTH * 16 * world,
                d2h=4 * world, loss=[loss_last])


def trained_state_leg(args, dev, stream, vp, vpi, tg, tuned, flush, retune=True):
    """The same step timed at a trained state: a fresh student of the same
    seed fitted for args.trained_steps steps with the plain ADC schedule
    (every 100 steps from 500 to 15k; the Gaussian count then differs from
    200k), then K steps timed exactly as the headline (CUDA events, L2
    flushed between steps)."""
    import torch

    from nprush_b200.gaussians import GaussianTrainer, random_gaussians
    from nprush_b200.train import AdcSchedule, evaluate_psnr, fit
    tr = GaussianTrainer(4 * N_GAUSS, sh_degree=SH_DEG, device=dev, params=random_gaussians(N_GAUSS, 10))
    tr.set_targets(tg, borrow=True)
    if tuned is not None:
        tr.set_tile(tuned["tile"])
        tr.set_raster((tuned["fwd_form"], tuned["fwd_ppt"], tuned["fwd_stage"]),
                      (tuned["bwd_form"], tuned["bwd_ppt"], tuned["bwd_stage"]))
    r = fit(tr, vp, vpi, args.trained_steps, views=VIEWS, seed=0,
            adc=AdcSchedule(stop=min(15000, args.trained_steps)))
    sched = view_schedule(args.warmup + args.steps)
    retuned = None
    if tuned is not None and retune:
        # the autotuner again, on the trained state (larger, more opaque Gaussians)
        tr.set_views(vp[sched[0]], vpi[sched[0]], sched[0])
        retuned = tr.autotune()
    tr.set_timing(not args.no_stage_timing)
    for k in range(args.warmup):
        tr.set_views(vp[sched[k]], vpi[sched[k]], sched[k])
        tr.train_step()
    torch.cuda.synchronize()
    tr.stage_times(reset=True)
    times, pairs = [], []
    for k in range(args.steps):
        sel = sched[args.warmup + k]
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tr.set_views(vp[sel], vpi[sel], sel)
        tr.train_step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        pairs.append(tr.stats()["pairs"])
    stages = tr.stage_times(reset=True)
    tr.set_timing(False)
    psnr = float(np.mean(evaluate_psnr(tr, vp, vpi)))
    out = {"after_steps": args.trained_steps, "gaussians": tr.count, "pairs_per_step": int(np.mean(pairs)),
           "ms_per_step": float(np.mean(times)), "steps_per_s": 1000.0 / float(np.mean(times)),
           "psnr_db": psnr, "fit_wall_s": r.wall_s, "fit_steps_per_s": args.trained_steps / r.wall_s,
           "stages_ms": {k: round(v[0] / max(v[1], 1), 4) for k, v in stages.items() if v[1]},
           "raster_variant": None if retuned is None else {k: v for k, v in retuned.items() if k != "per_tile"}}
    tr.close()
    return out


def cpu_baseline_port():
    """The oracle port of the same step on the host: one view of the workload
    (forward + loss + backward), plus Adam over all Gaussians, extrapolated to
    the 8-view step."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc  # checker / baseline only

    from nprush_b200.gaussians import orbit_cameras, random_gaussians, view_records
    vp, vpi = orbit_cameras(CAMS, WIDTH, HEIGHT)
    views = view_records(vp[:1], vpi[:1])
    teacher = random_gaussians(N_TEACHER, 11)
    timg, _ = orc.gs_forward(teacher, SH_DEG, views, WIDTH, HEIGHT)
    tg = timg.copy()
    tg[..., 3] = 1.0
    p = random_gaussians(N_GAUSS, 10)
    t0 = time.perf_counter()
    img, nc = orc.gs_forward(p, SH_DEG, views, WIDTH, HEIGHT)
    l3, dimg = orc.gs_loss(img, tg, np.zeros(1, np.uint32))
    g = orc.gs_backward(p, SH_DEG, views, WIDTH, HEIGHT, img, nc, dimg)
    t_view = time.perf_counter() - t0
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    t0 = time.perf_counter()
    orc.gs_adam(p, g, m, v, 1, (1.6e-4, 5e-3, 1e-3, 5e-2, 2.5e-3, 1.25e-4))
    t_adam = time.perf_counter() - t0
    step_s = VIEWS * t_view + t_adam
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"1 of 8 views of one step (fwd+loss+bwd {t_view:.2f} s) + Adam over all {N_GAUSS} "
                      f"Gaussians ({t_adam:.2f} s), extrapolated x8 views; fp32 C++ oracle, OpenMP"}


# ----------------------------------------------------------- reference arm
# The reference's own splat_backward.wgsl (translated to C++, oracle/_ref) is
# timed on every host core: a pool of processes (the translated shaders keep
# their workgroup runtime in process-global state), each loading the module
# and binding the same seeded inputs once, then running its share of a sample
# of 16 x 16 workgroups (tiles) spread evenly over the image.
_REF = {}


def _ref_splat_inputs(n):
    """The reference arm's seeded inputs at the headline shape: n splats of
    the reference's init distribution, one 800 x 800 target and depth."""
    from nprush_b200.gaussians import orbit_cameras
    rng = np.random.default_rng(10)
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    sc = np.exp(rng.normal(-4.0, 0.5, (n, 3)))
    s[:, 3], s[:, 12], s[:, 15] = sc[:, 0], sc[:, 1], sc[:, 2]
    s[:, 4:7] = rng.random((n, 3))
    s[:, 7] = np.clip(1 / (1 + np.exp(-rng.normal(0, 1, n))), 0.06, 0.99)
    q = rng.normal(size=(n, 4))
    s[:, 8:12] = q / np.linalg.norm(q, axis=1, keepdims=True)
    s[:, 13], s[:, 14] = 2.0, 0.5
    vp, vpi = orbit_cameras(CAMS, WIDTH, HEIGHT)
    tgt = np.zeros((HEIGHT, WIDTH, 4), np.float32)
    tgt[..., :3] = rng.random((HEIGHT, WIDTH, 3))
    dep = np.zeros((HEIGHT, WIDTH, 4), np.float32)
    dep[..., 0] = np.where(rng.random((HEIGHT, WIDTH)) < 0.5, 0.97, 1.0)
    uni = np.zeros(40, np.float32)
    uni[0:16], uni[16:32] = vp[0], vpi[0]
    return s, tgt, dep, uni


def _ref_worker_init(so_path, n):
    sys.path.insert(0, str(ROOT / "oracle"))
    import build_ref
    mod = build_ref.RefModule.from_path(so_path)
    s, tgt, dep, uni = _ref_splat_inputs(n)
    grads = np.zeros(n * 16, np.int32)
    mod.bind(0, s)
    mod.bind(1, grads)
    mod.bind_tex(2, tgt)
    mod.bind_tex(3, dep)
    mod.bind(4, uni)
    _REF["mod"] = mod


def _ref_worker_run(tiles, gx, gy):
    mod = _REF["mod"]
    for tx, ty in tiles:
        mod.run_one(tx, ty, 0, gx, gy, 1)
    return len(tiles)


def run_reference(args):
    """The reference's own splat_backward.wgsl + splat_step.wgsl (translated to
    C++ and compiled for the host, oracle/_ref) at this workload's shape:
    200k splats, 800x800, 8 views per step, on all host cores."""
    r = reference_splat_rate(args.steps)
    if "unavailable" in r:
        return {"impl": "reference", "unavailable": r["unavailable"]}
    v = r["value"]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "higher_is_better": True,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": "reference splat_backward + splat_step (its own WGSL, translated to C++) at the "
                                   "headline shape: 200k splats, 800x800, 8 views per step"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": r["cores"], "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_splat_rate(samples: int) -> dict:
    """Steps/s of the reference's splat_backward + splat_step at 200k splats,
    800x800, 8 views: each timed sample runs an evenly spread sample of the
    16x16 workgroups (tiles) of one view on a process pool over all host
    cores; the step time is the tile throughput extrapolated to every tile of
    the 8 views, plus one full splat_step dispatch."""
    import concurrent.futures as cf
    import multiprocessing as mp
    sys.path.insert(0, str(ROOT / "oracle"))
    import build_ref

    n = N_GAUSS
    so = sorted((ROOT / "oracle" / "_ref").glob(f"splat_backward_n{n}_*.so"))
    so_step = sorted((ROOT / "oracle" / "_ref").glob(f"splat_step_n{n}_*.so"))
    if not so or not so_step:
        if not build_ref.reference_available():
            return {"unavailable": "oracle/_ref for 200k splats was not built (no reference checkout)"}
        so = [build_ref.build("splat_backward", n)]
        so_step = [build_ref.build("splat_step", n)]
    gx, gy = (WIDTH + 15) // 16, (HEIGHT + 15) // 16
    workers = os.cpu_count() or 1
    # tiles on a regular lattice over the whole image (an unbiased sample of the tile costs)
    stride = 7
    tiles = [(x, y) for y in range(stride // 2, gy, stride) for x in range(stride // 2, gx, stride)]
    per_worker = max(1, -(-len(tiles) // workers))
    shares = [tiles[k:k + per_worker] for k in range(0, len(tiles), per_worker)]
    rates = []
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                initializer=_ref_worker_init, initargs=(str(so[-1]), n)) as ex:
        list(ex.map(_ref_worker_run, [shares[0][:1]] * workers, [gx] * workers, [gy] * workers))  # warm-up
        for _ in range(max(1, samples)):
            t0 = time.perf_counter()
            done = sum(ex.map(_ref_worker_run, shares, [gx] * len(shares), [gy] * len(shares)))
            rates.append(done / (time.perf_counter() - t0))
    tile_rate = float(np.median(rates))  # tiles per second over all workers
    s, _, _, _ = _ref_splat_inputs(n)
    mod_s = build_ref.RefModule.from_path(so_step[-1])
    grads = np.zeros(n * 16, np.int32)
    adam = np.zeros(32 * n + 8, np.float32)
    acc = np.zeros(n, np.float32)
    mod_s.bind(0, s)
    mod_s.bind(1, grads)
    mod_s.bind(2, adam)
    mod_s.bind(3, acc)
    t0 = time.perf_counter()
    mod_s.dispatch((n + 63) // 64, 1, 1)
    t_step = time.perf_counter() - t0
    step_s = gx * gy * VIEWS / tile_rate + t_step
    return {"value": 1.0 / step_s, "cores": workers,
            "sample": f"{len(tiles)} of {gx * gy} tiles of one view (a lattice, every {stride}th tile each way) per "
                      f"timed sample on {workers} processes ({tile_rate:.1f} tiles/s), extrapolated to {gx * gy} "
                      f"tiles x {VIEWS} views + one full splat_step ({t_step:.2f} s, one thread)"}


COMPAT_METRIC = ("splat optimiser dispatches/s (reference semantics: backward + step + ADC every 25th; 200k splats, "
                 "800^2, 8 views)")


def run_splat_compat(args):
    """The reference-semantics splat optimiser (nps_splat_opt_dispatch: the
    reference's splat_backward / splat_step / splat_adc, 1024 splats per tile,
    i32 fixed-point gradients) on the GPU at the reference arm's shape: the
    same 200k seeded splats and 800x800 target, 8 sphere cameras per
    dispatch.  CUDA events around each dispatch on the library's stream."""
    import torch

    from nprush_b200 import _lib
    from nprush_b200.gaussians import orbit_cameras
    from nprush_b200.splat import GpuSplatOptimizerManager
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    n = N_GAUSS
    s0, tgt, dep, _ = _ref_splat_inputs(n)
    vp, vpi = orbit_cameras(CAMS, WIDTH, HEIGHT)
    sel = view_schedule(1)[0]
    tg_host = np.ascontiguousarray(np.broadcast_to(tgt, (VIEWS,) + tgt.shape))
    dp_host = np.ascontiguousarray(np.broadcast_to(dep[..., 0], (VIEWS,) + dep.shape[:2]))
    with torch.cuda.stream(stream):
        m = GpuSplatOptimizerManager(n, device=dev, init=s0)
        m.write_splat_vp_matrix(vp[sel], vpi[sel])
        tg = torch.from_numpy(tg_host).cuda()
        dp = torch.from_numpy(dp_host).cuda()
        torch.cuda.synchronize()
        m.set_backward_target(tg, dp, WIDTH, HEIGHT, borrow=True)
        for _ in range(args.warmup):
            m.dispatch()
        flush = torch.empty(64 * 1024 * 1024, device=f"cuda:{dev}")
        times, bwd = [], []
        with ClockSampler(dev) as clk:
            for _ in range(args.steps):
                flush.zero_()
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(stream)
                m.dispatch()
                ev[1].record(stream)
                ev[1].synchronize()
                times.append(ev[0].elapsed_time(ev[1]))
            # the backward call alone (binning + the fused raster kernel), for the roofline
            for _ in range(args.steps):
                flush.zero_()
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(stream)
                m.backward()
                ev[1].record(stream)
                ev[1].synchronize()
                bwd.append(ev[0].elapsed_time(ev[1]))
        st = m.stats()
        # end to end: the caller's targets uploaded from page-locked host memory every dispatch
        host_t = torch.from_numpy(tg_host).pin_memory().numpy()
        host_d = torch.from_numpy(dp_host).pin_memory().numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            m.set_backward_target(host_t, host_d, WIDTH, HEIGHT)
            m.dispatch()
            m.sync()
        e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        m.close()
    ms = float(np.mean(times))
    ms_bwd = float(np.mean(bwd))
    pk, pk_kind = peaks()
    K = int(st["pairs_capped"])
    raster_bytes = K * (4 + 192) + VIEWS * WIDTH * HEIGHT * 36
    achieved = raster_bytes / (ms_bwd * 1e-3) / 1e9
    line = {
        "metric": COMPAT_METRIC, "value": 1000.0 / ms, "unit": "dispatches/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (i32 fixed-point gradients)",
        "data": "synthetic: the reference arm's seeded 200k splats and 800x800 target and depth",
        "config": {"workload": f"reference-semantics splat dispatch: {n // 1000}k splats, {WIDTH}x{HEIGHT}, "
                               f"{VIEWS} views per dispatch", "pairs_per_dispatch": int(st["pairs"]),
                   "pairs_composited": K, "max_tile_list": int(st["max_tile_len"]),
                   "l2": "flushed between timed dispatches (256 MB write)"},
        "clocks": clk.summary(),
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "dispatches/s",
                "h2d_bytes_per_step": VIEWS * WIDTH * HEIGHT * 20, "d2h_bytes_per_step": 0},
        "backward_ms": ms_bwd,
        "roofline": {"bound": "hbm", "kernel": "backward call (binning + compat::k_raster)", "achieved": achieved,
                     "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": None,
                     "peak_kind": pk_kind, "algorithmic_bytes": raster_bytes},
    }
    if not args.no_cpu_baseline:
        r = reference_splat_rate(3)
        if "value" in r:
            line["cpu_baseline"] = {"value": r["value"], "unit": "dispatches/s", "cores": r["cores"],
                                    "kind": "reference", "sample": r["sample"]}
    return line


# ------------------------------------------------- Bezier curve optimiser workload
BZ_N, BZ_TEACHER, BZ_RES, BZ_VIEWS, BZ_CAMS = 50_000, 60_000, 512, 4, 32
BZ_METRIC = ("Bezier optimiser dispatches/s (reference semantics: backward over 4 views + step + ADC every 50th; "
             "50k cubic curves, 512^2)")


def _bz_cameras():
    from nprush_b200.camera import sphere_cameras
    return sphere_cameras(BZ_CAMS, 4.0, math.radians(50.0), 1.0)


def run_bezier(args):
    """The reference-semantics Bezier optimiser (nps_bezier_opt_dispatch: the
    reference's bezier_backward / bezier_step / bezier_adc, 16-segment
    ribbons, 1024 curves per tile, i32 fixed-point gradients) on the GPU: 50k
    random-walk curves (seed 20) fitting the 512 x 512 renders of a seeded
    60k-curve teacher, 4 of 32 sphere cameras per dispatch.  CUDA events
    around each dispatch on the library's stream, L2 flushed between them."""
    import torch

    from nprush_b200 import _lib
    from nprush_b200.bezier import GpuBezierOptimizerManager
    from nprush_b200.bezier_fit import random_walk_curves
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    W = H = BZ_RES
    V = BZ_VIEWS
    vp, vpi = _bz_cameras()
    rng = np.random.default_rng(5)
    sels = [np.sort(rng.permutation(BZ_CAMS)[:V]) for _ in range(args.warmup + 2 * args.steps)]
    with torch.cuda.stream(stream):
        teacher = GpuBezierOptimizerManager(BZ_TEACHER, init=random_walk_curves(BZ_TEACHER, 21, H))
        tg = torch.zeros((BZ_CAMS, H, W, 4), device="cuda")
        for c in range(BZ_CAMS):
            teacher.render(vp[c], W, H, tg[c])
        teacher.close()
        m = GpuBezierOptimizerManager(BZ_N, init=random_walk_curves(BZ_N, 20, H))
        m.write_mode(1.0)
        depth = torch.ones((V, H, W, 4), device="cuda")
        zeros = torch.zeros((V, H, W, 4), device="cuda")
        tgs = [tg[torch.as_tensor(sel, device="cuda")].contiguous() for sel in sels]

        def step(k):
            m.write_vp(vp[sels[k]], vpi[sels[k]])
            m.set_backward_target(tgs[k], depth, zeros, depth, zeros, W, H, borrow=True)
            m.dispatch()

        for k in range(args.warmup):
            step(k)
        flush = torch.empty(64 * 1024 * 1024, device=f"cuda:{dev}")
        times = []
        with ClockSampler(dev) as clk:
            for k in range(args.steps):
                flush.zero_()
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(stream)
                step(args.warmup + k)
                ev[1].record(stream)
                ev[1].synchronize()
                times.append(ev[0].elapsed_time(ev[1]))
        st = m.stats()
        # end to end: the caller's four targets (rgba + depth, background, normals) from page-locked host memory
        host = [torch.from_numpy(tgs[0].cpu().numpy()).pin_memory().numpy()]
        hd, hz = (torch.from_numpy(x.cpu().numpy()).pin_memory().numpy() for x in (depth, zeros))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.steps):
            m.write_vp(vp[sels[args.warmup + args.steps + k]], vpi[sels[args.warmup + args.steps + k]])
            m.set_backward_target(host[0], hd, hz, hd, hz, W, H)
            m.dispatch()
            _lib.call("nps_sync", ctx)
        e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        m.close()
    ms = float(np.mean(times))
    line = {
        "metric": BZ_METRIC, "value": 1000.0 / ms, "unit": "dispatches/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (i32 fixed-point gradients)",
        "data": "synthetic: seeded random-walk curves; targets rendered from a seeded 60k-curve teacher",
        "config": {"workload": f"reference-semantics Bezier dispatch: {BZ_N // 1000}k cubic curves, {W}x{H}, "
                               f"{V} of {BZ_CAMS} sphere cameras per dispatch, ADC every 50th",
                   "pairs_per_dispatch": int(st["pairs"]), "l2": "flushed between timed dispatches (256 MB write)"},
        "clocks": clk.summary(),
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "dispatches/s",
                "h2d_bytes_per_step": int(host[0].nbytes + 4 * hd.nbytes), "d2h_bytes_per_step": 0},
    }
    if not args.no_cpu_baseline:
        r = reference_bezier_rate(3)
        if "value" in r:
            line["cpu_baseline"] = {"value": r["value"], "unit": "dispatches/s", "cores": r["cores"],
                                    "kind": "reference", "sample": r["sample"]}
    return line


def _bz_ref_worker_init(so_path, n):
    sys.path.insert(0, str(ROOT / "oracle"))
    import build_ref
    import refrun
    from nprush_b200.bezier_fit import random_walk_curves
    mod = build_ref.RefModule.from_path(so_path)
    vp, vpi = _bz_cameras()
    rng = np.random.default_rng(11)
    tgt = np.zeros((BZ_RES, BZ_RES, 4), np.float32)
    tgt[..., :3] = rng.random((BZ_RES, BZ_RES, 3))
    tgt[..., 3] = 1.0
    one = np.zeros((BZ_RES, BZ_RES, 4), np.float32)
    one[..., 0] = 1.0
    zero = np.zeros((BZ_RES, BZ_RES, 4), np.float32)
    keep = [random_walk_curves(n, 20, BZ_RES), np.zeros(n * 18, np.int32), tgt, one,
            refrun.bezier_uniforms(vp[0], vpi[0], mode=1.0), zero, one, np.zeros(2 * n, np.float32), zero,
            np.zeros(512 * 512, np.int32)]
    for slot, a in enumerate(keep):
        (mod.bind_tex if slot in (2, 3, 5, 6, 8) else mod.bind)(slot, a)
    _REF["bz"] = (mod, keep)


def _bz_ref_worker_run(tiles, gx, gy):
    mod = _REF["bz"][0]
    for tx, ty in tiles:
        mod.run_one(tx, ty, 0, gx, gy, 1)
    return len(tiles)


def reference_bezier_rate(samples: int) -> dict:
    """Dispatches/s of the reference's bezier_backward + bezier_step at 50k
    curves, 512 x 512, 4 views per dispatch (the reference fits one view per
    backward dispatch, so one of these dispatches is 4 of its backward
    dispatches and one step): each timed sample runs a lattice of the 16 x 16
    workgroups of one view on a process pool over all host cores; the
    dispatch time is the tile throughput extrapolated to every tile of the 4
    views, plus one full bezier_step dispatch.  ADC (every 50th) not counted."""
    import concurrent.futures as cf
    import multiprocessing as mp
    sys.path.insert(0, str(ROOT / "oracle"))
    import build_ref

    n = BZ_N
    so = sorted((ROOT / "oracle" / "_ref").glob(f"bezier_backward_n{n}_*.so"))
    so_step = sorted((ROOT / "oracle" / "_ref").glob(f"bezier_step_n{n}_*.so"))
    if not so or not so_step:
        if not build_ref.reference_available():
            return {"unavailable": "oracle/_ref for 50k curves was not built (no reference checkout)"}
        so = [build_ref.build("bezier_backward", n)]
        so_step = [build_ref.build("bezier_step", n)]
    gx = gy = (BZ_RES + 15) // 16
    workers = os.cpu_count() or 1
    stride = 5
    tiles = [(x, y) for y in range(stride // 2, gy, stride) for x in range(stride // 2, gx, stride)]
    per_worker = max(1, -(-len(tiles) // workers))
    shares = [tiles[k:k + per_worker] for k in range(0, len(tiles), per_worker)]
    rates = []
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                initializer=_bz_ref_worker_init, initargs=(str(so[-1]), n)) as ex:
        list(ex.map(_bz_ref_worker_run, [shares[0][:1]] * workers, [gx] * workers, [gy] * workers))  # warm-up
        for _ in range(max(1, samples)):
            t0 = time.perf_counter()
            done = sum(ex.map(_bz_ref_worker_run, shares, [gx] * len(shares), [gy] * len(shares)))
            rates.append(done / (time.perf_counter() - t0))
    tile_rate = float(np.median(rates))
    from nprush_b200.bezier_fit import random_walk_curves
    import refrun
    vp, vpi = _bz_cameras()
    mod_s = build_ref.RefModule.from_path(so_step[-1])
    b = random_walk_curves(n, 20, BZ_RES)
    adam = np.zeros(36 * n + 8, np.float32)
    adam[36 * n + 1] = 1.0
    arrs = [b, np.zeros(n * 18, np.int32), adam, np.zeros(2 * n, np.float32),
            refrun.bezier_uniforms(vp[0], vpi[0], mode=1.0)]
    for slot, a in enumerate(arrs):
        mod_s.bind(slot, a)
    t0 = time.perf_counter()
    mod_s.dispatch((n + 63) // 64, 1, 1)
    t_step = time.perf_counter() - t0
    disp_s = gx * gy * BZ_VIEWS / tile_rate + t_step
    return {"value": 1.0 / disp_s, "cores": workers,
            "sample": f"{len(tiles)} of {gx * gy} tiles of one view (a lattice, every {stride}th tile each way) per "
                      f"timed sample on {workers} processes ({tile_rate:.1f} tiles/s), extrapolated to {gx * gy} "
                      f"tiles x {BZ_VIEWS} views + one full bezier_step ({t_step:.3f} s, one thread); ADC not "
                      "counted; random target (its values do not change the per-pixel work)"}


def run_bezier_reference(args):
    r = reference_bezier_rate(args.steps)
    if "unavailable" in r:
        return {"impl": "reference", "unavailable": r["unavailable"]}
    v = r["value"]
    return {"impl": "reference", "metric": BZ_METRIC, "value": v, "unit": "dispatches/s", "higher_is_better": True,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": "reference bezier_backward + bezier_step (its own WGSL, translated to C++): "
                                   "50k cubic curves, 512x512, 4 views per dispatch"},
            "cpu_baseline": {"value": v, "unit": "dispatches/s", "cores": r["cores"], "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": "dispatches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


METRIC = "train steps/s (fwd+bwd+Adam, 200k splats, 800^2, 8 views)"
FWD_FORMS = ("one CTA per (tile, view)", "persistent warp-specialised, longest-first queue",
             "one CTA per (tile, view), longest first")
BWD_FORMS = FWD_FORMS

# ------------------------------------------------- path-traced target workload
PT_W, PT_H, PT_OBJECTS, PT_DETAIL, PT_BATCH = 1024, 768, 16, 20, 8
PT_METRIC = "path-traced samples/s (1 sample per pixel per frame, <= 8 bounces, 12k-triangle scene, 1024x768)"


def pt_scene():
    from nprush_b200 import camera, meshes
    sc = meshes.demo_scene(PT_OBJECTS, seed=7, mirror_fraction=0.3, sphere_detail=PT_DETAIL)
    env = meshes.sky_env(256, 128)
    _, inv = camera.view_proj((4.0, -3.5, 2.6), (0.0, 0.0, 0.3), 0.9, PT_W / PT_H, up=(0.0, 0.0, 1.0))
    return sc, env, inv


def pt_reference_sample(args):
    """The reference's own path_trace.wgsl (translated to C++, oracle/_ref) on
    the host: a spread of its 8 x 8 workgroups of one frame, extrapolated to
    the frame.  Returns (samples/s, description) or (None, why)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import build_ref
    sc, env, inv = pt_scene()
    so = sorted((ROOT / "oracle" / "_ref").glob("path_trace_n0_*.so"))
    if not so and not build_ref.reference_available():
        return None, "oracle/_ref path_trace was not built (no reference checkout)"
    from bvh import build_bvh
    nodes, tris = build_bvh(sc.vertices, sc.indices)
    mod = build_ref.RefModule.from_path(so[-1]) if so else build_ref.RefModule("path_trace", 0)
    acc = np.zeros((PT_H, PT_W, 4), np.float32)
    uni = np.zeros(20, np.uint32)
    uni[:16] = np.ascontiguousarray(inv, np.float32).view(np.uint32)
    uni[16:20] = [0, tris.shape[0], PT_W, PT_H]
    mod.bind(0, uni)
    mod.bind(1, np.ascontiguousarray(sc.vertices, np.float32).reshape(-1))
    mod.bind(2, np.ascontiguousarray(nodes).reshape(-1))
    mod.bind(3, np.ascontiguousarray(tris).reshape(-1))
    mod.bind(4, acc)
    mod.bind_tex(5, env)
    mod.bind_sampler(6, True, "repeat", "clamp-to-edge")
    gx, gy = PT_W // 8, PT_H // 8
    groups = [(x, y) for y in range(3, gy, 11) for x in range(5, gx, 13)]
    per = []
    for _ in range(max(1, min(args.steps, 5))):
        t0 = time.perf_counter()
        for x, y in groups:
            mod.run_one(x, y, 0, gx, gy, 1)
        per.append((time.perf_counter() - t0) / (len(groups) * 64))
    t_sample = float(np.median(per))
    return 1.0 / t_sample, (f"{len(groups)} of {gx * gy} 8x8 workgroups of one frame per timed sample "
                            f"({t_sample * 1e6:.1f} us per path), extrapolated; single host thread")


MR_W, MR_H, MR_OBJECTS, MR_DETAIL = 1024, 768, 40, 32
MR_METRIC = "mesh render passes/s (environment + ~80k-triangle mesh, colour + reciprocal depth targets, 1024x768)"


def mr_scene():
    from nprush_b200 import camera, meshes
    sc = meshes.demo_scene(MR_OBJECTS, seed=7, mirror_fraction=0.0, sphere_detail=MR_DETAIL)
    eye, tgt = (4.0, -3.5, 2.6), (0.0, 0.0, 0.3)
    vp, inv = camera.view_proj(eye, tgt, 0.9, MR_W / MR_H, up=(0.0, 0.0, 1.0))
    u = np.zeros(52, np.float32)
    u[0:16], u[16:32], u[36:52] = vp, camera.col_major(camera.look_at(eye, tgt, (0.0, 0.0, 1.0))), inv
    return sc, meshes.sky_env(256, 128), u


def mr_cpu_sample(stages_for):
    """Host timing of the mesh pass on the same scene through oracle/mesh_raster.py
    with the stage functions stages_for(uniforms, env) returns: one pass at
    64x48 and one at 128x96, fitted as t = a + b * pixels (a: the per-vertex and
    per-triangle work, b: the per-pixel work) and evaluated at the workload's
    1024x768.  Returns (passes/s, description)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import mesh_raster as mr
    from nprush_b200 import camera
    sc, env, uni = mr_scene()
    ts = {}
    for w, h in ((64, 48), (128, 96)):
        su = uni.copy()
        vp, inv = camera.view_proj((4.0, -3.5, 2.6), (0.0, 0.0, 0.3), 0.9, w / h, up=(0.0, 0.0, 1.0))
        su[0:16], su[36:52] = vp, inv
        stages = stages_for(su, env)
        t0 = time.perf_counter()
        mr.render(sc.vertices, sc.indices, su, w, h, stages)
        ts[w * h] = time.perf_counter() - t0
    (p0, t0_), (p1, t1_) = sorted(ts.items())
    b = max((t1_ - t0_) / (p1 - p0), 0.0)
    a = max(t0_ - b * p0, 0.0)
    t_full = a + b * MR_W * MR_H
    return 1.0 / t_full, (f"passes at 64x48 ({t0_:.1f} s) and 128x96 ({t1_:.1f} s) fitted as {a:.1f} s + "
                          f"{b * 1e6:.1f} us per pixel, evaluated at {MR_W}x{MR_H} ({t_full:.0f} s); one host thread")


def run_mesh_raster(args):
    """The viewer's mesh render pass (nps_mesh_render): CUDA events around
    each pass on the library's stream; the CPU leg is the float32 restatement
    (oracle/mesh_raster.py) at 64 x 48 on the same scene, per pixel scaled."""
    import torch

    from nprush_b200 import _lib
    from nprush_b200.mesh_render import MeshRenderer
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    sc, env, uni = mr_scene()
    with torch.cuda.stream(stream):
        r = MeshRenderer(sc, matcap=env, env=env, device=dev)
        r.uniforms[:] = uni
        col = torch.empty((MR_H, MR_W, 4), dtype=torch.float32, device=f"cuda:{dev}")
        dep = torch.empty_like(col)
        torch.cuda.synchronize()

        def one():
            _lib.call("nps_mesh_render", r._h, r.uniforms.ctypes.data, col.data_ptr(), dep.data_ptr(), MR_W, MR_H,
                      1, 1)

        for _ in range(args.warmup):
            one()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        with ClockSampler(dev) as clk:
            ev[0].record(stream)
            for _ in range(args.steps):
                one()
            ev[1].record(stream)
            ev[1].synchronize()
        ms = ev[0].elapsed_time(ev[1]) / args.steps
        host_c = torch.empty((MR_H, MR_W, 4), dtype=torch.float32, pin_memory=True)
        host_d = torch.empty_like(host_c)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            one()
            host_c.copy_(col, non_blocking=True)
            host_d.copy_(dep, non_blocking=True)
            stream.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        r.close()
    line = {
        "metric": MR_METRIC, "value": 1000.0 / ms, "unit": "passes/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: seeded ground + 40 spheres and boxes, procedural sky and matcap",
        "config": {"workload": f"mesh render pass: {sc.n_tris} triangles, {MR_W}x{MR_H}, 8-bit targets",
                   "triangles": sc.n_tris, "resolution": [MR_W, MR_H]},
        "clocks": clk.summary(),
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "passes/s", "h2d_bytes_per_step": 208,
                "d2h_bytes_per_step": 2 * MR_W * MR_H * 16},
        "gpu_launches": 7 * args.steps,  # vertex, setup, 3 scan passes, raster, shade
        "roofline": None,
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import mesh_raster as mr
        v, why = mr_cpu_sample(lambda su, env_: mr.RestatedStages(env_, env_))
        line["cpu_baseline"] = {"value": v, "unit": "passes/s", "cores": 1, "kind": "port",
                                "sample": "the float32 restatement (numpy): " + why}
    return line


def mr_reference(args):
    """The reference's own mesh.wgsl / envmap.wgsl stage functions (translated
    to C++, oracle/_ref) between the restated fixed-function steps, on the
    host; its render pipeline itself needs a graphics stack, which this box
    does not have."""
    sys.path.insert(0, str(ROOT / "oracle"))
    try:
        import refrun
        refrun.stage_module("mesh")
    except FileNotFoundError as e:
        return {"impl": "reference", "unavailable": str(e)}
    v, why = mr_cpu_sample(lambda su, env_: refrun.MeshStages(su, env_, env_))
    return {"impl": "reference", "metric": MR_METRIC, "value": v, "unit": "passes/s", "higher_is_better": True,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": "reference mesh.wgsl / envmap.wgsl stages (translated to C++) with the restated "
                                   "fixed-function steps, same scene"},
            "cpu_baseline": {"value": v, "unit": "passes/s", "cores": 1, "kind": "reference", "sample": why},
            "e2e": {"value": v, "unit": "passes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_path_trace(args):
    import torch

    from nprush_b200 import _lib
    from nprush_b200.path_trace import PathTracer
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = _lib.context(dev)
    _lib.call("nps_set_stream", ctx, stream.cuda_stream)
    sc, env, inv = pt_scene()
    with torch.cuda.stream(stream):
        pt = PathTracer(env_texture=env, device=dev)
        pt.set_meshes(sc)
        pt.set_output_size(PT_W, PT_H)
        pt.write_inv_view_proj_mat(inv)
        torch.cuda.synchronize()

        def timed(frames_per_launch, launches):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            for _ in range(launches):
                pt.trace(frames_per_launch)
            ev[1].record(stream)
            ev[1].synchronize()
            return ev[0].elapsed_time(ev[1])

        timed(1, args.warmup)
        with ClockSampler(dev) as clk:
            ms = timed(1, args.steps)
            ms_batch = timed(PT_BATCH, max(1, args.steps // PT_BATCH))
        # end to end through the public API: the camera matrix goes up with
        # the launch, the resolved 8-bit image comes back to the host
        host = torch.empty((PT_H, PT_W, 4), dtype=torch.float32, pin_memory=True)
        pt.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pt.write_inv_view_proj_mat(inv)
            pt.dispatch(frames=1, sync=False)
            host.copy_(pt.output, non_blocking=True)
            stream.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        overflows = pt.overflows()
        pt.close()
    npx = PT_W * PT_H
    ms_step = ms / args.steps
    line = {
        "metric": PT_METRIC, "value": npx / (ms_step * 1e-3), "unit": "samples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded ground + 16 spheres and boxes (30% mirrors), procedural sky environment",
        "config": {"workload": f"path-traced targets: {sc.n_tris} triangles, {PT_W}x{PT_H}, one frame per step",
                   "triangles": sc.n_tris, "resolution": [PT_W, PT_H], "l2": "scene resident (BVH < L2)",
                   "batched": {"frames_per_launch": PT_BATCH,
                               "samples_per_s": npx * PT_BATCH * max(1, args.steps // PT_BATCH) / (ms_batch * 1e-3)}},
        "clocks": clk.summary(),
        "e2e": {"value": npx / (e2e_ms * 1e-3), "unit": "samples/s", "h2d_bytes_per_step": 64,
                "d2h_bytes_per_step": npx * 16},
        "gpu_launches": args.steps,
        "roofline": None,
        "bound": "latency / issue (divergent BVH traversal; the BVH and vertices sit in L2)",
        "traversal_overflows": overflows,
    }
    if not args.no_cpu_baseline:
        v, why = pt_reference_sample(args)
        line["cpu_baseline"] = (None if v is None else
                                {"value": v, "unit": "samples/s", "cores": 1, "kind": "reference", "sample": why})
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="train", choices=["train", "splat_compat", "bezier", "path_trace", "mesh_raster"],
                    help="train: the Gaussian train step (headline); splat_compat: the reference-semantics splat "
                         "optimiser at the reference arm's shape; path_trace: path-traced target generation; "
                         "mesh_raster: the viewer's mesh render pass (colour + depth targets)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # smaller shapes for profiler captures (the bench number is the 200k / 800x800 workload only)
    ap.add_argument("--gaussians", type=int, default=None)
    ap.add_argument("--res", type=int, default=None)
    ap.add_argument("--views", type=int, default=None)
    ap.add_argument("--no-flush", action="store_true", help="do not flush L2 between timed steps")
    ap.add_argument("--no-stage-timing", action="store_true", help="no per-stage CUDA events")
    ap.add_argument("--no-graph", action="store_true", help="launch the step eagerly instead of as a CUDA graph")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default raster variants")
    ap.add_argument("--raster", default=None,
                    help="fixed tile and raster variants instead of the autotuner: "
                         "tile,fwd_form,fwd_ppt,fwd_stage,bwd_form,bwd_ppt,bwd_stage")
    ap.add_argument("--trained-steps", type=int, default=15000,
                    help="also time the step after fitting a fresh student this many steps (0: skip)")
    args = ap.parse_args()
    global N_GAUSS, N_TEACHER, WIDTH, HEIGHT, VIEWS
    if args.gaussians:
        N_GAUSS, N_TEACHER = args.gaussians, args.gaussians * 5 // 4
    if args.res:
        WIDTH = HEIGHT = args.res
    if args.views:
        VIEWS = args.views
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.workload == "mesh_raster":
        if rank == 0:
            print(json.dumps(mr_reference(args) if args.impl == "reference" else run_mesh_raster(args)))
        return
    if args.workload == "splat_compat":
        if rank == 0:
            if args.impl == "reference":
                r = run_reference(args)
                if "metric" in r:
                    r["metric"], r["unit"] = COMPAT_METRIC, "dispatches/s"
                    r["e2e"]["unit"] = r["cpu_baseline"]["unit"] = "dispatches/s"
                print(json.dumps(r))
            else:
                print(json.dumps(run_splat_compat(args)))
        return
    if args.workload == "bezier":
        if rank == 0:
            print(json.dumps(run_bezier_reference(args) if args.impl == "reference" else run_bezier(args)))
        return
    if args.workload == "path_trace":
        if rank != 0:
            return
        if args.impl == "reference":
            v, why = pt_reference_sample(args)
            line = ({"impl": "reference", "unavailable": why} if v is None else
                    {"impl": "reference", "metric": PT_METRIC, "value": v, "unit": "samples/s",
                     "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                     "config": {"workload": "reference path_trace.wgsl (translated to C++) on the same scene"},
                     "cpu_baseline": {"value": v, "unit": "samples/s", "cores": 1, "kind": "reference", "sample": why},
                     "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        else:
            line = run_path_trace(args)
        print(json.dumps(line))
        return
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_sharded(args, rank, world) if world > 1 else run_ours(args, rank, world)
    ms = res["ms_total"]
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    ms_per_step = ms / args.steps
    strong = res.get("scaling") == "strong"
    value = (1.0 if strong else world) * 1000.0 / ms_per_step
    pk, pk_kind = peaks()
    npx = WIDTH * HEIGHT
    K = res["pairs"]
    tile = res["tuned"]["tile"] if res.get("tuned") else 16
    tile_passes = int(math.ceil(math.ceil(math.log2(VIEWS * (-(-WIDTH // tile)) * (-(-HEIGHT // tile)))) / 8))
    st = res["stages"]
    if not any(v[1] for v in st.values()):
        st = {k: (1.0, 1) for k in st}  # stage timing disabled
    dom = max(st, key=lambda k: st[k][0])
    dom_ms = st[dom][0] / max(st[dom][1], 1)
    v_local = res.get("views_local", VIEWS)  # views this rank rendered per step
    achieved = stage_bytes(dom, v_local, N_GAUSS, K, npx, tile_passes) / (dom_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if strong else "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded 200k-Gaussian student, targets rendered from a seeded 250k-Gaussian teacher",
        "config": {"workload": (f"{N_GAUSS // 1000}k Gaussians SH3, {WIDTH}x{HEIGHT}, {VIEWS} of {CAMS} "
                                "sphere cameras per step, L1 + 0.2 D-SSIM, Adam"), "gaussians": N_GAUSS, "resolution": [WIDTH, HEIGHT],
                   "views_per_step": VIEWS,
                   "l2": "not flushed" if args.no_flush else "flushed between timed steps (256 MB write)",
                   "pairs_per_step": K, "parallelism": (f"view-sharded over {world} GPUs (NCCL all-reduce of the gradients per step)"
                                   if world > 1 else "single GPU"),
                   "cuda_graph": not args.no_graph and world == 1,
                   "raster_variant": (None if res.get("tuned") is None else
                                      {"tile": res["tuned"]["tile"],
                                       "fwd_form": FWD_FORMS[res["tuned"]["fwd_form"]],
                                       "bwd_form": BWD_FORMS[res["tuned"]["bwd_form"]],
                                       "per_tile": res["tuned"]["per_tile"],
                                       "fwd_pixels_per_thread": res["tuned"]["fwd_ppt"],
                                       "fwd_records_per_stage": res["tuned"]["fwd_stage"],
                                       "bwd_pixels_per_thread": res["tuned"]["bwd_ppt"],
                                       "bwd_records_per_stage": res["tuned"]["bwd_stage"],
                                       "chosen_by": "autotuner"})},
        "clocks": res["clocks"],
        "e2e": {"value": (1.0 if strong else world) * 1000.0 / res["e2e_ms"], "unit": "steps/s",
                "h2d_bytes_per_step": res["h2d"],
                "d2h_bytes_per_step": res["d2h"]},
        "gpu_launches": None if res["graph_kernels"] is None else res["graph_kernels"] * args.steps,
        "gpu_launches_source": "kernel nodes of the captured train-step graph x timed steps",
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"], "traffic": (BWD_TRAFFIC_BYTES * K / BWD_TRAFFIC_PAIRS
                                 if dom == "raster_bwd" and N_GAUSS == 200_000 and WIDTH == 800 else None),
                     "traffic_source": "ncu capture of the same kernel and workload, scaled by pairs",
                     "peak_kind": pk_kind,
                     "step_algorithmic_bytes": step_bytes(VIEWS, N_GAUSS, K, npx),
                     "step_frac": step_bytes(VIEWS, N_GAUSS, K, npx) / (ms_per_step * 1e-3) / 1e9 / pk["hbm_gbs"],
                     "issue": {k: issue_roofline(k, res.get("tuned"), K, st[k][0] / max(st[k][1], 1),
                                                 (res["clocks"] or {}).get("sm_mhz"))
                               for k in ("raster_fwd", "raster_bwd") if k in st}},
        "stages_ms": {k: round(v[0] / max(v[1], 1), 4) for k, v in st.items()},
        "trained_state": res["trained"],
        "final_loss": res["loss"],
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port()
    print(json.dumps(line))


if __name__ == "__main__":
    main()
