"""3D Gaussian trainer over libnprush_cuda (3D Gaussians with SH colour).

Keeps the reference's fit-a-scene call pattern (GpuSplatOptimizerManager:
write params -> write camera(s) -> set target(s) -> dispatch), for standard
3D Gaussians with SH colour, batched over many views per call, plus the paired
forward / backward entry points.

Parameter record (64 floats): mean xyz, log-scale xyz, quaternion wxyz,
opacity logit, pad, 16 x rgb SH coefficients (coefficient-major), pad.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import NPS_MEM_HOST, call
from .splat import _ptr

P = 64
SH_C0 = 0.28209479177387814
PARAM_FIELDS = {"mean": slice(0, 3), "log_scale": slice(3, 6), "quat": slice(6, 10), "opacity": slice(10, 11),
                "sh": slice(12, 60)}


def random_gaussians(n: int, seed: int, sh_degree: int = 3, sh_rest_std: float = 0.1) -> np.ndarray:
    """Seeded scene: means U[-1,1]^3, log-scales N(-4, 0.5), random unit
    quaternions, opacity logits N(0,1), RGB U[0,1] as SH DC, higher SH N(0, std)."""
    rng = np.random.default_rng(seed)
    p = np.zeros((n, P), np.float32)
    p[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    p[:, 3:6] = rng.normal(-4.0, 0.5, (n, 3))
    q = rng.normal(size=(n, 4))
    p[:, 6:10] = q / np.linalg.norm(q, axis=1, keepdims=True)
    p[:, 10] = rng.normal(0, 1, n)
    rgb = rng.random((n, 3))
    p[:, 12:15] = (rgb - 0.5) / SH_C0
    nb = (sh_degree + 1) ** 2
    if nb > 1:
        p[:, 15:12 + 3 * nb] = rng.normal(0, sh_rest_std, (n, 3 * (nb - 1)))
    return p


def view_records(vp, vp_inv) -> np.ndarray:
    """The 48-float per-view record the kernels use: vp, vp_inv, camera centre."""
    vp = np.asarray(vp, np.float32).reshape(-1, 16)
    vpi = np.asarray(vp_inv, np.float32).reshape(-1, 16)
    out = np.zeros((vp.shape[0], 48), np.float32)
    out[:, :16] = vp
    out[:, 16:32] = vpi
    c = vpi[:, 8:12].astype(np.float64)
    out[:, 32:35] = (c[:, :3] / c[:, 3:4]).astype(np.float32)
    return out


class GaussianTrainer:
    LR_DEFAULT = (1.6e-4, 5e-3, 1e-3, 5e-2, 2.5e-3, 2.5e-3 / 20)

    def __init__(self, capacity: int, sh_degree: int = 3, device: int = 0, params=None, lr=None):
        self.capacity = int(capacity)
        self.sh_degree = int(sh_degree)
        self.device = device
        self._ctx = _lib.context(device)
        h = ctypes.c_void_p()
        call("nps_gs_create", self._ctx, self.capacity, self.sh_degree, ctypes.byref(h))
        self._h = h.value
        self.count = 0
        self._keep = []
        if params is not None:
            self.write_params(params)
        self.set_lr(lr or self.LR_DEFAULT)

    def write_params(self, params, first: int = 0):
        p, mem, keep = _ptr(params)
        n = (keep.numel() if mem != NPS_MEM_HOST else keep.size) // P
        call("nps_gs_write_params", self._h, p, first, n, mem)
        self.count = max(self.count, first + n)

    def set_count(self, n: int):
        call("nps_gs_set_count", self._h, n)
        self.count = n

    def set_lr(self, lr6):
        a = np.ascontiguousarray(lr6, np.float32)
        call("nps_gs_set_lr", self._h, a.ctypes.data)

    def set_background(self, rgb):
        call("nps_gs_set_background", self._h, float(rgb[0]), float(rgb[1]), float(rgb[2]))

    def set_targets(self, rgba, borrow: bool = False):
        """rgba: T x H x W x 4 float images (numpy or torch CUDA)."""
        t, h, w = rgba.shape[0], rgba.shape[1], rgba.shape[2]
        p, mem, keep = _ptr(rgba, borrow=borrow)
        call("nps_gs_set_targets", self._h, p, w, h, t, mem)
        self._keep = [keep] if borrow else []
        self.width, self.height = w, h

    def upload_targets(self, host_images, ids):
        """Targets = host_images[ids] (numpy [T, H, W, 4] float32, page-locked for
        overlap, e.g. a pinned torch tensor's .numpy()), copied on a side stream
        and put in place after the steps already queued."""
        a = host_images
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"] and a.ndim == 4
        ids = np.ascontiguousarray(ids, np.uint32)
        call("nps_gs_upload_targets", self._h, a.ctypes.data, ids.ctypes.data, len(ids), a.shape[2], a.shape[1])
        self.width, self.height = a.shape[2], a.shape[1]

    def read_loss(self):
        l3 = np.zeros(3, np.float32)
        call("nps_gs_read_loss", self._h, l3.ctypes.data)
        return tuple(float(x) for x in l3)

    def set_image_size(self, width: int, height: int):
        call("nps_gs_set_image_size", self._h, width, height)
        self.width, self.height = width, height

    def set_views(self, vp, vp_inv, target_ids=None):
        vp = np.ascontiguousarray(vp, np.float32).reshape(-1, 16)
        vpi = np.ascontiguousarray(vp_inv, np.float32).reshape(-1, 16)
        ids = None
        if target_ids is not None:
            ids = np.ascontiguousarray(target_ids, np.uint32)
        call("nps_gs_set_views", self._h, vp.ctypes.data, vpi.ctypes.data, None if ids is None else ids.ctypes.data,
             vp.shape[0])
        self.num_views = vp.shape[0]

    def forward(self, out=None):
        """Renders all views; out: optional torch CUDA tensor [V,H,W,4] (rgb, T)."""
        p = None
        if out is not None:
            import torch
            torch.cuda.current_stream(out.device).synchronize()
            p = out.data_ptr()
        call("nps_gs_forward", self._h, p)
        if out is not None:
            self.sync()

    def loss(self, read_back: bool = True):
        l3 = np.zeros(3, np.float32)
        call("nps_gs_loss", self._h, l3.ctypes.data if read_back else None)
        return tuple(float(x) for x in l3) if read_back else None

    LOSS_KINDS = {"l1_dssim": 0, "l1": 1, "l2": 2}

    def set_loss(self, kind: str = "l1_dssim", ssim_weight: float = 0.2):
        """Loss of the fused path: "l1_dssim" ((1 - w) L1 + w D-SSIM), "l1" or "l2"."""
        call("nps_gs_set_loss", self._h, self.LOSS_KINDS[kind], float(ssim_weight))

    def backward(self, dl_dimage=None):
        """dl_dimage: None (the fused loss's gradient), a torch CUDA tensor or
        a numpy array [V,H,W,4] (copied from host memory)."""
        if isinstance(dl_dimage, np.ndarray):
            a = np.ascontiguousarray(dl_dimage, np.float32)
            call("nps_gs_backward_host", self._h, a.ctypes.data)
            return
        p = None
        if dl_dimage is not None:
            import torch
            torch.cuda.current_stream(dl_dimage.device).synchronize()
            p = dl_dimage.data_ptr()
        call("nps_gs_backward", self._h, p)

    def adam(self):
        call("nps_gs_adam", self._h)

    def set_graph(self, enable: bool):
        """Capture the train step as one CUDA graph after the first call."""
        call("nps_gs_set_graph", self._h, int(bool(enable)))

    def train_step(self, read_loss: bool = False):
        l3 = np.zeros(3, np.float32)
        call("nps_gs_train_step", self._h, l3.ctypes.data if read_loss else None)
        return tuple(float(x) for x in l3) if read_loss else None

    def read_state(self):
        n = self.count
        out = {k: np.empty((n, P), np.float32) for k in ("params", "grads", "adam_m", "adam_v")}
        ag = np.empty(n, np.float32)
        ad = np.empty(n, np.float32)
        call("nps_gs_read_state", self._h, out["params"].ctypes.data, out["grads"].ctypes.data,
             out["adam_m"].ctypes.data, out["adam_v"].ctypes.data, ag.ctypes.data, ad.ctypes.data)
        out["adc_grad"], out["adc_denom"] = ag, ad
        return out

    def write_state(self, adam_m=None, adam_v=None, step: int = 0):
        m, mem, k1 = _ptr(adam_m)
        v, mem2, k2 = _ptr(adam_v)
        call("nps_gs_write_state", self._h, m, v, int(step), mem if adam_m is not None else mem2)

    VARIANTS = ((1, 256), (2, 128), (2, 256), (4, 64), (4, 128))  # form 0 (16 x 16 tiles): one CTA per (tile, view)
    # form 1: persistent, warp-specialised, per tile edge
    PERSISTENT_VARIANTS = {8: ((1, 64), (1, 128), (2, 64), (2, 128)),
                           16: ((1, 128), (2, 64), (2, 128), (4, 64), (4, 128)),
                           32: ((4, 64), (4, 128))}
    TUNE_VARIANTS = (tuple((0,) + v for v in VARIANTS) + ((1, 1, 64), (1, 1, 128), (1, 2, 64), (1, 2, 128),
                                                          (1, 4, 64), (1, 4, 128)) + tuple((2,) + v for v in VARIANTS))

    def set_variant(self, fwd_ppt: int, bwd_ppt: int, fwd_stage: int = 0, bwd_stage: int = 0):
        """Form-0 raster kernels with 1, 2 or 4 pixels per thread and the given
        records staged per batch (0: 256 / pixels per thread)."""
        call("nps_gs_set_variant", self._h, int(fwd_ppt), int(fwd_stage), int(bwd_ppt), int(bwd_stage))

    def set_raster(self, fwd=(0, 1, 256), bwd=(0, 2, 128)):
        """(form, pixels per thread, records per stage) of the forward and the
        backward raster; form 1 is the persistent warp-specialised kernel,
        form 2 one CTA per tile taking the tiles longest first."""
        call("nps_gs_set_raster", self._h, *[int(x) for x in fwd], *[int(x) for x in bwd])

    def set_tile(self, tile: int):
        """Tile edge of the binning and raster (8, 16 or 32)."""
        call("nps_gs_set_tile", self._h, int(tile))

    def raster(self) -> dict:
        c = np.zeros(7, np.int32)
        call("nps_gs_get_raster", self._h, c.ctypes.data)
        return dict(tile=int(c[0]), fwd=tuple(int(x) for x in c[1:4]), bwd=tuple(int(x) for x in c[4:7]))

    def autotune(self, cache_path=None) -> dict:
        """Times binning at every tile size and the raster variants of both
        forms of each tile on the current views / targets; keeps the fastest
        (looked up in / appended to cache_path when given)."""
        nv = len(self.TUNE_VARIANTS)
        c = np.zeros(7, np.int32)
        t = np.zeros(3 * (1 + 2 * nv), np.float32)
        call("nps_gs_autotune_raster", self._h, None if cache_path is None else str(cache_path).encode(),
             c.ctypes.data, t.ctypes.data)
        per_tile = {}
        for k, tile in enumerate((8, 16, 32)):
            row = t[(1 + 2 * nv) * k:(1 + 2 * nv) * (k + 1)]
            per_tile[tile] = dict(binning_ms=float(row[0]), fwd_ms=row[1:1 + nv].tolist(),
                                  bwd_ms=row[1 + nv:1 + 2 * nv].tolist())
        return dict(tile=int(c[0]), fwd_form=int(c[1]), fwd_ppt=int(c[2]), fwd_stage=int(c[3]),
                    bwd_form=int(c[4]), bwd_ppt=int(c[5]), bwd_stage=int(c[6]), per_tile=per_tile,
                    cached=bool(t[0] < 0))

    def set_sort_guard(self, spin_limit: int = 0, stall_tile: int = 0xFFFFFFFF):
        """Look-back bound of the onesweep sorts (0: the default); stall_tile
        (tests) is a tile whose status is treated as never published."""
        call("nps_gs_set_sort_guard", self._h, int(spin_limit), int(stall_tile))

    def set_deterministic(self, enable: bool):
        """Two-pass backward reduction without float atomics (bit-reproducible)."""
        call("nps_gs_set_deterministic", self._h, int(bool(enable)))

    def set_accumulate(self, accumulate: bool, loss_views: int = 0):
        call("nps_gs_set_accumulate", self._h, int(bool(accumulate)), int(loss_views))

    def train_step_per_view(self, vp, vp_inv, target_ids, read_loss: bool = False):
        """One step of the plain per-view trainer: the step's V views are
        rendered, differentiated and accumulated one launch at a time (eager),
        then one Adam update.  Same gradient as train_step over the V views."""
        vp = np.asarray(vp, np.float32).reshape(-1, 16)
        vpi = np.asarray(vp_inv, np.float32).reshape(-1, 16)
        ids = np.ascontiguousarray(target_ids, np.uint32)
        nv = vp.shape[0]
        total = np.zeros(3, np.float64)
        l3 = np.zeros(3, np.float32)
        for k in range(nv):
            self.set_accumulate(k > 0, nv)
            self.set_views(vp[k:k + 1], vpi[k:k + 1], ids[k:k + 1])
            call("nps_gs_forward", self._h, None)
            call("nps_gs_loss", self._h, l3.ctypes.data if read_loss else None)
            total += l3
            call("nps_gs_backward", self._h, None)
        call("nps_gs_adam", self._h)
        self.set_accumulate(False, 0)
        if read_loss:
            # each view's terms are its share of the V-view means: they sum to them
            return tuple(float(x) for x in total)
        return None

    def save(self, path):
        """Checkpoint: parameters, Adam state and step, ADC accumulators."""
        call("nps_gs_save", self._h, str(path).encode())

    def load(self, path):
        call("nps_gs_load", self._h, str(path).encode())
        self.count = self._count()

    def _count(self) -> int:
        c = ctypes.c_uint32()
        call("nps_gs_count", self._h, ctypes.byref(c))
        return int(c.value)

    def write_adc_stats(self, adc_grad, adc_denom):
        g, mem, k1 = _ptr(adc_grad)
        d, mem2, k2 = _ptr(adc_denom)
        assert mem == mem2
        call("nps_gs_write_adc_stats", self._h, g, d, mem)

    def adc(self, grad_thresh: float = 2e-4, split_scale: float = 0.01, prune_opacity: float = 0.005) -> dict:
        """Densify (clone / split) and prune; returns the counts."""
        c = np.zeros(4, np.uint32)
        call("nps_gs_adc", self._h, float(grad_thresh), float(split_scale), float(prune_opacity), c.ctypes.data)
        self.count = int(c[1])
        return dict(before=int(c[0]), after=int(c[1]), densified=int(c[2]), pruned=int(c[3]))

    def assign_ids(self, base: int = 0):
        """Lineage ids (record float 63) = base + index; inherited by clones / children."""
        call("nps_gs_assign_ids", self._h, int(base))

    def adc_features(self, step_frac: float, grad_thresh: float = 2e-4, split_scale: float = 0.01,
                     prune_opacity: float = 0.005):
        """(features [n,16] f32, plain decision [n] u8, lineage id [n] i32) as torch CUDA tensors."""
        import torch
        n = self.count
        dev = f"cuda:{self.device}"
        feat = torch.empty((max(n, 1), 16), device=dev, dtype=torch.float32)
        plain = torch.empty(max(n, 1), device=dev, dtype=torch.uint8)
        ids = torch.empty(max(n, 1), device=dev, dtype=torch.int32)
        call("nps_gs_adc_features", self._h, float(step_frac), float(grad_thresh), float(split_scale),
             float(prune_opacity), feat.data_ptr(), plain.data_ptr(), ids.data_ptr())
        self.sync()
        return feat[:n], plain[:n], ids[:n]

    def set_policy_margin(self, margin: float):
        """Keep's logit in the policy decision (0 = argmax; > 0 acts only when confident)."""
        call("nps_gs_set_policy_margin", self._h, float(margin))

    def adc_policy(self, policy, step_frac: float, grad_thresh: float = 2e-4, split_scale: float = 0.01,
                   prune_opacity: float = 0.005) -> dict:
        """ADC decided by the policy network (None: the plain rule)."""
        c = np.zeros(4, np.uint32)
        fb = ctypes.c_uint32(0)
        call("nps_gs_adc_policy", self._h, None if policy is None else policy._h, float(step_frac),
             float(grad_thresh), float(split_scale), float(prune_opacity), c.ctypes.data, ctypes.byref(fb))
        self.count = int(c[1])
        return dict(before=int(c[0]), after=int(c[1]), densified=int(c[2]), pruned=int(c[3]), fallback=int(fb.value))

    def psnr(self):
        """Per-view PSNR (dB) of the last forward."""
        out = np.zeros(self.num_views, np.float32)
        call("nps_gs_psnr", self._h, out.ctypes.data)
        return out

    def read_image(self, with_grad: bool = True):
        """(image [V,H,W,4], dL/dimage [V,H,W,4] or None) of the last forward / loss."""
        shape = (self.num_views, self.height, self.width, 4)
        img = np.empty(shape, np.float32)
        dimg = np.empty(shape, np.float32) if with_grad else None
        call("nps_gs_read_image", self._h, img.ctypes.data, None if dimg is None else dimg.ctypes.data)
        return img, dimg

    def buffers(self) -> dict:
        ptrs = [ctypes.c_void_p() for _ in range(6)]
        call("nps_gs_buffers", self._h, *[ctypes.byref(p) for p in ptrs])
        return dict(zip(("params", "grads", "adam_m", "adam_v", "image", "dl_dimage"), [p.value for p in ptrs]))

    def adc_buffers(self) -> dict:
        ptrs = [ctypes.c_void_p() for _ in range(2)]
        call("nps_gs_adc_buffers", self._h, *[ctypes.byref(p) for p in ptrs])
        return dict(adc_grad=ptrs[0].value, adc_denom=ptrs[1].value)

    def stats(self) -> dict:
        st = _lib.nps_stats()
        call("nps_gs_stats", self._h, ctypes.byref(st))
        return dict(pairs=st.pairs, step_count=st.step_count, graph_kernels=st.reserved[0],
                    skipped_steps=st.reserved[1], staging_timeouts=st.reserved[2])

    STAGES = ("preprocess", "depth_sort", "emit", "tile_sort", "ranges", "raster_fwd", "loss", "raster_bwd",
              "project_bwd", "adam")

    def set_timing(self, enable: bool):
        call("nps_gs_set_timing", self._h, int(bool(enable)))

    def stage_times(self, reset: bool = True) -> dict:
        """{stage: (total ms, launches)} since the last reset."""
        ms = np.zeros(len(self.STAGES), np.float64)
        calls = np.zeros(len(self.STAGES), np.uint64)
        call("nps_gs_stage_times", self._h, ms.ctypes.data, calls.ctypes.data, len(self.STAGES), int(reset))
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(self.STAGES)}

    def sync(self):
        call("nps_sync", self._ctx)

    def close(self):
        if getattr(self, "_h", None):
            call("nps_gs_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def orbit_cameras(n: int = 32, width: int = 800, height: int = 800, fov_deg: float = 50.0, radius: float = 4.0):
    from .camera import sphere_cameras
    return sphere_cameras(n, radius, math.radians(fov_deg), width / height)
