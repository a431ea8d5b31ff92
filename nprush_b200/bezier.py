"""Python mirror of the reference's Bezier optimiser over libnprush_cuda.

GpuBezierOptimizerManager  <->  src/lib/gpu/GpuBezierOptimizerManager.ts
    constructor({numBeziers})            -> GpuBezierOptimizerManager(num_beziers=...)
    writeVPMatrix / writeVPInvMatrix     -> write_vp_matrix / write_vp_inv_matrix
    writeMode, writeBgPenalty, writeMaxWidth, writeKillThresholds,
    setAdcPeriod, writeNoKill            -> same names in snake_case
    setBackwardTarget(t, td, bg, bgd, n, w, h) -> set_backward_target(...)
    dispatch(encoder)                    -> dispatch()
Errors raise NpsError (the reference reports them asynchronously).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import NPS_MEM_DEVICE_BORROW, NPS_MEM_HOST, call
from .splat import _ptr

FLOATS_PER_BEZIER = 20
PARAMS_PER_BEZIER = 18
PIXEL_LOSS_SIZE = 512 * 512


def reference_init(num_beziers: int, seed: int = 0) -> np.ndarray:
    """Seeded version of the reference's initial curves
    (GpuBezierOptimizerManager.ts:60-95): short random squiggles near the origin."""
    rng = np.random.default_rng(seed)
    n = num_beziers
    b = np.zeros((n, 20), np.float32)
    cx, cy = rng.random(n) * 2 - 1, rng.random(n) * 2 - 1
    ln = 0.2 + rng.random(n) * 0.2
    ang = rng.random(n) * math.pi * 2
    dx, dy = np.cos(ang) * ln, np.sin(ang) * ln
    jit = lambda: (rng.random(n) - 0.5) * 0.08  # noqa: E731
    b[:, 0], b[:, 1], b[:, 2], b[:, 3] = cx - dx * 0.5, cy - dy * 0.5, (rng.random(n) * 2 - 1) * 0.3, 0.02
    b[:, 4], b[:, 5], b[:, 6], b[:, 7] = cx - dx * 0.15 + jit(), cy - dy * 0.15 + jit(), (rng.random(n) * 2 - 1) * 0.3, 0.005
    b[:, 8], b[:, 9], b[:, 10] = cx + dx * 0.15 + jit(), cy + dy * 0.15 + jit(), (rng.random(n) * 2 - 1) * 0.3
    b[:, 12], b[:, 13], b[:, 14] = cx + dx * 0.5, cy + dy * 0.5, (rng.random(n) * 2 - 1) * 0.3
    b[:, 16:19] = rng.random((n, 3))
    b[:, 19] = 0.5
    return b


class GpuBezierOptimizerManager:
    def __init__(self, num_beziers: int = 16, device: int = 0, init=None, seed: int = 0):
        self.num_beziers = int(num_beziers)
        self.num_params = self.num_beziers * PARAMS_PER_BEZIER
        self._ctx = _lib.context(device)
        h = ctypes.c_void_p()
        call("nps_bezier_opt_create", self._ctx, self.num_beziers, ctypes.byref(h))
        self._h = h.value
        self._keep = []
        self._vp = self._vp_inv = None  # last matrices written (host copies)
        if init is None:
            init = reference_init(self.num_beziers, seed)
        if init is not False:
            self.write_params(init)

    def write_params(self, beziers, first: int = 0):
        p, mem, keep = _ptr(beziers)
        count = (keep.numel() if mem != NPS_MEM_HOST else keep.size) // FLOATS_PER_BEZIER
        call("nps_bezier_opt_write_params", self._h, p, first, count, mem)

    def write_state(self, grads=None, adam_m=None, adam_v=None, adam_t=0.0, grad_accum=None, loss_accum=None,
                    pixel_loss=None):
        ptrs = []
        keep = []
        for a, dt in ((grads, np.int32), (adam_m, np.float32), (adam_v, np.float32), (grad_accum, np.float32),
                      (loss_accum, np.float32), (pixel_loss, np.int32)):
            p, _, k = _ptr(a, dt)
            ptrs.append(p)
            keep.append(k)
        call("nps_bezier_opt_write_state", self._h, ptrs[0], ptrs[1], ptrs[2], ctypes.c_float(adam_t), ptrs[3],
             ptrs[4], ptrs[5], NPS_MEM_HOST)

    def read_state(self):
        n = self.num_beziers
        out = dict(beziers=np.empty((n, 20), np.float32), grads=np.empty((n, 18), np.int32),
                   adam_m=np.empty((n, 18), np.float32), adam_v=np.empty((n, 18), np.float32),
                   grad_accum=np.empty(n, np.float32), loss_accum=np.empty(n, np.float32),
                   pixel_loss=np.empty(PIXEL_LOSS_SIZE, np.int32))
        t = ctypes.c_float()
        call("nps_bezier_opt_read_state", self._h, out["beziers"].ctypes.data, out["grads"].ctypes.data,
             out["adam_m"].ctypes.data, out["adam_v"].ctypes.data, ctypes.byref(t), out["grad_accum"].ctypes.data,
             out["loss_accum"].ctypes.data, out["pixel_loss"].ctypes.data)
        out["adam_t"] = t.value
        return out

    # ---- reference API
    def write_vp(self, vp, vp_inv):
        """Both matrices at once ([V,]16 each, one pair per view)."""
        vp = np.ascontiguousarray(vp, np.float32).reshape(-1, 16)
        vpi = np.ascontiguousarray(vp_inv, np.float32).reshape(-1, 16)
        if vp.shape != vpi.shape:
            raise ValueError("vp and vp_inv must have the same number of views")
        call("nps_bezier_opt_write_vp", self._h, vp.ctypes.data, vpi.ctypes.data, vp.shape[0])
        self._vp, self._vp_inv = vp.copy(), vpi.copy()

    def write_vp_matrix(self, mat):
        """writeVPMatrix (GpuBezierOptimizerManager.ts:269-277): the view-projection
        alone.  The inverse keeps its last value; one never written reads as
        zeros, as in the reference's zero-initialised uniform buffer (also when
        the number of views changes, until write_vp_inv_matrix follows)."""
        vp = np.ascontiguousarray(mat, np.float32).reshape(-1, 16)
        vpi = self._vp_inv
        if vpi is None or vpi.shape != vp.shape:
            vpi = np.zeros_like(vp)
        self.write_vp(vp, vpi)

    def write_vp_inv_matrix(self, mat):
        """writeVPInvMatrix (GpuBezierOptimizerManager.ts:279-288): the inverse
        alone, the view-projection kept (zeros if never written)."""
        vpi = np.ascontiguousarray(mat, np.float32).reshape(-1, 16)
        vp = self._vp
        if vp is None or vp.shape != vpi.shape:
            vp = np.zeros_like(vpi)
        self.write_vp(vp, vpi)

    def write_mode(self, mode: float = 0.0):
        call("nps_bezier_opt_write_mode", self._h, float(mode))

    def write_bg_penalty(self, weight: float = 0.0):
        call("nps_bezier_opt_write_bg_penalty", self._h, float(weight))

    def write_max_width(self, max_width: float = 0.0):
        call("nps_bezier_opt_write_max_width", self._h, float(max_width))

    def write_kill_thresholds(self, alpha_thresh: float = 0.0, width_thresh: float = 0.0):
        call("nps_bezier_opt_write_kill_thresholds", self._h, float(alpha_thresh), float(width_thresh))

    def set_adc_period(self, period: int):
        call("nps_bezier_opt_set_adc_period", self._h, int(period))

    def write_no_kill(self, no_kill: bool):
        call("nps_bezier_opt_write_no_kill", self._h, int(bool(no_kill)))

    def set_backward_target(self, target, target_depth, bg, bg_depth, normal, width: int, height: int,
                            borrow: bool = False):
        shape = tuple(target.shape)
        views = 1 if len(shape) == 3 else shape[0]
        ps, keep = [], []
        mem = NPS_MEM_HOST
        for a in (target, target_depth, bg, bg_depth, normal):
            p, m, k = _ptr(a, borrow=borrow)
            ps.append(p)
            keep.append(k)
            mem = m
        call("nps_bezier_opt_set_target", self._h, *ps, width, height, views, mem)
        self._keep = keep if borrow else []

    def dispatch(self):
        call("nps_bezier_opt_dispatch", self._h)

    def backward(self, out_rgbd=None):
        p = None
        if out_rgbd is not None:
            import torch
            torch.cuda.current_stream(out_rgbd.device).synchronize()
            p = out_rgbd.data_ptr()
        call("nps_bezier_opt_backward", self._h, p)
        if out_rgbd is not None:
            call("nps_sync", self._ctx)

    def render(self, vp, width: int, height: int, out, background=None, brush=None):
        """Headless GpuBezierForwardPipelineManager.dispatch: out (torch CUDA
        [H,W,4]) receives the premultiplied composite over `background`
        (torch CUDA [H,W,4] or None = cleared); brush: torch CUDA [bh,bw]."""
        import torch
        torch.cuda.current_stream(out.device).synchronize()
        vp = np.ascontiguousarray(vp, np.float32).reshape(16)
        bgp = background.data_ptr() if background is not None else None
        brp, bw, bh = (None, 0, 0) if brush is None else (brush.data_ptr(), brush.shape[1], brush.shape[0])
        call("nps_bezier_opt_render", self._h, vp.ctypes.data, width, height, bgp, brp, bw, bh, out.data_ptr())
        call("nps_sync", self._ctx)

    def step(self):
        call("nps_bezier_opt_step", self._h)

    def adc(self):
        call("nps_bezier_opt_adc", self._h)

    def stats(self) -> dict:
        st = _lib.nps_stats()
        call("nps_bezier_opt_stats", self._h, ctypes.byref(st))
        return dict(pairs=st.pairs, adc_clones=st.adc_clones, spawns=st.reserved[0], step_count=st.step_count)

    def set_step_count(self, count: int):
        """stepCount (dispatch() calls so far; ADC every adc_period)."""
        call("nps_bezier_opt_set_step_count", self._h, int(count))

    def close(self):
        if getattr(self, "_h", None):
            call("nps_bezier_opt_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # camelCase aliases (the reference's method names)
    writeVPMatrix = write_vp_matrix
    writeVPInvMatrix = write_vp_inv_matrix
    writeMode = write_mode
    writeBgPenalty = write_bg_penalty
    writeMaxWidth = write_max_width
    writeKillThresholds = write_kill_thresholds
    setAdcPeriod = set_adc_period
    writeNoKill = write_no_kill
    setBackwardTarget = set_backward_target


class GpuBezierForwardPipelineManager:
    """GpuBezierForwardPipelineManager (src/lib/gpu/GpuBezierForwardPipelineManager.ts),
    headless: draws the curves of an optimiser's bezierBuffer into one RGBA
    image.  The reference's constructor({device, numBeziers, bezierBuffer,
    brushTexture}) takes the optimiser's buffer and the brush texture
    (GpuRunner.svelte.ts:210-229); here the optimiser and the brush as a torch
    CUDA [bh, bw] float32 image (None: analytic coverage only)."""

    def __init__(self, optimizer: GpuBezierOptimizerManager, brush=None):
        self._opt = optimizer
        self._brush = brush
        self._vp = np.zeros(16, np.float32)  # the uniform buffer starts zeroed
        self._target = None

    def write_vp_matrix(self, mat):
        """writeVPMatrix (:102-110)."""
        self._vp = np.ascontiguousarray(mat, np.float32).reshape(16).copy()

    def set_target(self, target, width: int, height: int):
        """setTarget(view, w, h) (:112-129): a torch CUDA float32 [H,W,4] image."""
        if tuple(target.shape) != (height, width, 4):
            raise ValueError(f"target shape {tuple(target.shape)} does not match {height}x{width}x4")
        self._target = (target, int(width), int(height))

    def dispatch(self, clear: bool = True):
        """dispatch(encoder, clear) (:131-148): clear = cleared to 0 first;
        otherwise the curves are composited over the image's current contents
        (the render pass's "load")."""
        if self._target is None:
            raise _lib.NpsError(-6, "bezier forward dispatch: no target (set_target first)")
        out, w, h = self._target
        background = None if clear else out.clone()
        self._opt.render(self._vp, w, h, out, background=background, brush=self._brush)

    writeVPMatrix = write_vp_matrix
    setTarget = set_target
