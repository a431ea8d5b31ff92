"""Python mirror of the reference's splat manager classes over libnprush_cuda.

GpuSplatOptimizerManager  <->  src/lib/gpu/GpuSplatOptimizerManager.ts
    constructor({numSplats})        -> GpuSplatOptimizerManager(num_splats=...)
    writeSplatVPMatrix(vp, vpInv)   -> write_splat_vp_matrix(vp, vp_inv)
    setBackwardTarget(c, d, w, h)   -> set_backward_target(rgba, depth, w, h)
    dispatch(encoder)               -> dispatch()
    setEdgeTarget(depth, edge)      -> set_edge_target(depth, edge)
    dispatchEdge(encoder, w, h)     -> dispatch_edge(w, h)
Same names (camelCase aliases included), same argument meaning; the reference
reports errors asynchronously and silently skips dispatch without a target
(GpuSplatOptimizerManager.ts:366) — here every call raises NpsError instead.

Arrays may be numpy (host; copied) or torch CUDA tensors (device; copied, or
borrowed with borrow=True like a texture view bound into a bind group).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import NPS_MEM_DEVICE, NPS_MEM_DEVICE_BORROW, NPS_MEM_HOST, call

FLOATS_PER_SPLAT = 16


def _ptr(a, dtype=np.float32, borrow=False):
    """(pointer, mem kind, keepalive) for a numpy array or torch tensor."""
    if a is None:
        return None, NPS_MEM_HOST, None
    try:
        import torch
        if isinstance(a, torch.Tensor):
            if not a.is_cuda:
                a = a.detach().cpu().numpy()
            else:
                # the library runs on its own stream: make torch's producers finish first
                torch.cuda.current_stream(a.device).synchronize()
                want = {np.float32: torch.float32, np.int32: torch.int32}[dtype]
                if a.dtype != want or not a.is_contiguous():
                    if borrow:
                        raise ValueError("borrowed tensors must be contiguous and of the right dtype")
                    a = a.to(want).contiguous()
                return a.data_ptr(), (NPS_MEM_DEVICE_BORROW if borrow else NPS_MEM_DEVICE), a
    except ImportError:
        pass
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data, NPS_MEM_HOST, arr


def reference_init(num_splats: int, seed: int = 0) -> np.ndarray:
    """Seeded version of the reference's initial splats
    (GpuSplatOptimizerManager.ts:58-86): 512 live splats near the origin."""
    rng = np.random.default_rng(seed)
    s = np.zeros((num_splats, 16), np.float32)
    s[:, 0:3] = (rng.random((num_splats, 3)) * 2 - 1) * 0.3
    s[:, 3] = 0.1 + rng.random(num_splats) * 0.15
    s[:, 4:7] = rng.random((num_splats, 3))
    live = min(num_splats, 512)
    s[:live, 7] = 0.3 + rng.random(live) * 0.4
    s[:, 8] = 1.0
    s[:, 12] = 0.1 + rng.random(num_splats) * 0.15
    s[:, 13] = 2.0
    s[:, 14] = 0.5
    s[:, 15] = 0.1 + rng.random(num_splats) * 0.15
    return s


class GpuSplatOptimizerManager:
    """Reference-semantics splat trainer (fixed-point gradients, index-order
    compositing, 1024-per-tile cap, Adam with box clamps, serial-equivalent ADC)."""

    ADC_PERIOD = 25  # GpuSplatOptimizerManager.ts:381

    def __init__(self, num_splats: int = 512, device: int = 0, init=None, seed: int = 0):
        self.device = device
        self.num_splats = int(num_splats)
        self.num_params = self.num_splats * 16
        self._ctx = _lib.context(device)
        h = ctypes.c_void_p()
        call("nps_splat_opt_create", self._ctx, self.num_splats, ctypes.byref(h))
        self._h = h.value
        self._keep = []
        self._edge = None
        self.dims = (0, 0)
        if init is None:
            init = reference_init(self.num_splats, seed)
        if init is not False:
            self.write_params(init)

    # ---- buffers
    def write_params(self, splats, first: int = 0):
        """queue.writeBuffer(splatBuffer, first * 64, splats)."""
        p, mem, keep = _ptr(splats)
        count = (keep.numel() if mem != NPS_MEM_HOST else keep.size) // FLOATS_PER_SPLAT
        call("nps_splat_opt_write_params", self._h, p, first, count, mem)

    def write_state(self, adam_m=None, adam_v=None, adam_t: float = 0.0, grad_accum=None, grads=None):
        """Adam m / v, step counter, grad_accum and the i32 gradient buffer
        (host arrays; None leaves a buffer unchanged)."""
        pq, _, kq = _ptr(grads, np.int32)
        pm, _, km = _ptr(adam_m)
        pv, _, kv = _ptr(adam_v)
        pg, _, kg = _ptr(grad_accum)
        call("nps_splat_opt_write_state", self._h, pq, pm, pv, ctypes.c_float(adam_t), pg, NPS_MEM_HOST)

    def read_state(self):
        n = self.num_splats
        s = np.empty((n, 16), np.float32)
        g = np.empty((n, 16), np.int32)
        m = np.empty((n, 16), np.float32)
        v = np.empty((n, 16), np.float32)
        ga = np.empty(n, np.float32)
        t = ctypes.c_float()
        call("nps_splat_opt_read_state", self._h, s.ctypes.data, g.ctypes.data, m.ctypes.data, v.ctypes.data,
             ctypes.byref(t), ga.ctypes.data)
        return dict(splats=s, grads=g, adam_m=m, adam_v=v, adam_t=t.value, grad_accum=ga)

    def read_params(self) -> np.ndarray:
        s = np.empty((self.num_splats, 16), np.float32)
        call("nps_splat_opt_read_state", self._h, s.ctypes.data, None, None, None, None, None)
        return s

    def buffers(self) -> dict:
        """Device pointers of splatBuffer, gradBuffer, Adam m/v and grad_accum."""
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        call("nps_splat_opt_buffers", self._h, *[ctypes.byref(p) for p in ptrs])
        return dict(zip(("splats", "grads", "adam_m", "adam_v", "grad_accum"), [p.value for p in ptrs]))

    # ---- reference API
    def write_splat_vp_matrix(self, vp, vp_inv, blur_enabled: bool = False):
        vp = np.ascontiguousarray(vp, np.float32).reshape(-1, 16)
        vpi = np.ascontiguousarray(vp_inv, np.float32).reshape(-1, 16)
        if vp.shape != vpi.shape:
            raise ValueError("vp and vp_inv must have the same number of views")
        call("nps_splat_opt_write_vp", self._h, vp.ctypes.data, vpi.ctypes.data, vp.shape[0], int(bool(blur_enabled)))

    def set_backward_target(self, rgba, depth, width: int, height: int, borrow: bool = False):
        """rgba: [V,]H,W,4 floats (.rgb used); depth: [V,]H,W floats."""
        shape = tuple(rgba.shape)
        views = 1 if len(shape) == 3 else shape[0]
        if shape[-3:] != (height, width, 4):
            raise ValueError(f"target shape {shape} does not match {height}x{width}x4")
        pr, mem, kr = _ptr(rgba, borrow=borrow)
        pd, _, kd = _ptr(depth, borrow=borrow)
        call("nps_splat_opt_set_target", self._h, pr, pd, width, height, views, mem)
        self._keep = [kr, kd] if borrow else []
        self.dims = (width, height)

    def dispatch(self):
        call("nps_splat_opt_dispatch", self._h)

    def set_edge_target(self, depth, edge):
        """setEdgeTarget(depthView, edgeView) (GpuSplatOptimizerManager.ts:319-328):
        binds a depth image and the edge image that dispatch_edge writes, both
        torch CUDA float32 [H,W,4] tensors (depth in channel 0), held like the
        texture views of a bind group."""
        if tuple(depth.shape) != tuple(edge.shape):
            raise ValueError(f"depth {tuple(depth.shape)} and edge {tuple(edge.shape)} images differ in shape")
        self._edge = (depth, edge)

    def dispatch_edge(self, width: int, height: int, quantize: bool = True):
        """dispatchEdge(encoder, width, height) (GpuSplatOptimizerManager.ts:390-400):
        the Sobel depth-edge pass (splat_edge.wgsl) over the bound images.  The
        reference dispatches ceil(w/16) x ceil(h/16) workgroups and the shader
        stops at the depth texture's size; its viewer always passes that size
        (GpuRunner.svelte.ts:686, :760), and a dispatch that does not cover the
        image is refused here.  quantize: the edge texture is rgba8unorm."""
        from . import targets
        edge = self._edge
        if edge is None:
            raise _lib.NpsError(-6, "dispatch_edge: no edge target (set_edge_target first)")
        depth, out = edge
        h, w = int(depth.shape[0]), int(depth.shape[1])
        if (int(width) + 15) // 16 * 16 < w or (int(height) + 15) // 16 * 16 < h:
            raise ValueError(f"dispatch_edge({width}, {height}) does not cover the {w}x{h} edge target")
        targets.splat_edge(depth, out, quantize=quantize)

    # ---- the three stages of dispatch, separately
    def backward(self, out_rgbd=None):
        """splat_backward over all views; out_rgbd: optional torch CUDA tensor
        [V,H,W,4] receiving the fp32 composite (r, g, b, reciprocal depth)."""
        p = None
        if out_rgbd is not None:
            import torch
            torch.cuda.current_stream(out_rgbd.device).synchronize()
            p = out_rgbd.data_ptr()
        call("nps_splat_opt_backward", self._h, p)
        if out_rgbd is not None:
            self.sync()  # torch reads the image on its own stream

    def render(self, vp, width: int, height: int, out_rgba, out_depth=None, load: bool = False):
        """Headless GpuSplatForwardPipelineManager.dispatch(enc, clear=not load):
        out_rgba / out_depth: torch CUDA [H,W,4] float tensors, cleared first
        or, with load=True, blended over in place."""
        import torch
        torch.cuda.current_stream(out_rgba.device).synchronize()
        for t in (out_rgba, out_depth):
            if t is not None and (tuple(t.shape) != (height, width, 4) or t.dtype != torch.float32
                                  or not t.is_cuda or not t.is_contiguous()):
                raise ValueError(f"render target must be a contiguous CUDA float32 [{height},{width},4] tensor")
        vp = np.ascontiguousarray(vp, np.float32).reshape(16)
        call("nps_splat_opt_render_load" if load else "nps_splat_opt_render", self._h, vp.ctypes.data, width, height,
             out_rgba.data_ptr(), None if out_depth is None else out_depth.data_ptr())
        self.sync()

    def step(self):
        call("nps_splat_opt_step", self._h)

    def adc(self):
        call("nps_splat_opt_adc", self._h)

    def stats(self) -> dict:
        st = _lib.nps_stats()
        call("nps_splat_opt_stats", self._h, ctypes.byref(st))
        return dict(pairs=st.pairs, pairs_capped=st.pairs_capped, max_tile_len=st.max_tile_len,
                    adc_clones=st.adc_clones, step_count=st.step_count, pairs_kept=st.reserved[1],
                    timeouts=st.reserved[2])

    def set_wait_guard(self, spin_limit: int = 0, stall_batch: int = 0xFFFFFFFF):
        """Polls before a raster staging wait gives up (0: the default);
        stall_batch (tests) is a batch of tile 0 whose copies are never
        issued, so its wait runs out."""
        call("nps_splat_opt_set_wait_guard", self._h, int(spin_limit), int(stall_batch))

    def set_step_count(self, count: int):
        """stepCount (dispatch() calls so far; ADC every 25th)."""
        call("nps_splat_opt_set_step_count", self._h, int(count))

    def sync(self):
        call("nps_sync", self._ctx)

    def close(self):
        if getattr(self, "_h", None):
            call("nps_splat_opt_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # camelCase aliases (the reference's method names)
    writeSplatVPMatrix = write_splat_vp_matrix
    setBackwardTarget = set_backward_target
    setEdgeTarget = set_edge_target
    dispatchEdge = dispatch_edge


class GpuSplatForwardPipelineManager:
    """GpuSplatForwardPipelineManager (src/lib/gpu/GpuSplatForwardPipelineManager.ts),
    headless: draws the splats of an optimiser's splatBuffer into a colour and
    a depth image.  The reference's constructor({device, numSplats,
    splatBuffer}) takes the optimiser's buffer (GpuRunner.svelte.ts:204-208);
    here the optimiser itself."""

    def __init__(self, optimizer: GpuSplatOptimizerManager):
        self._opt = optimizer
        self._vp = np.zeros(16, np.float32)  # the uniform buffer starts zeroed
        self._target = None

    def write_vp_matrix(self, mat):
        """writeVPMatrix (:94-102)."""
        self._vp = np.ascontiguousarray(mat, np.float32).reshape(16).copy()

    def set_target(self, color, depth, width: int, height: int):
        """setTarget(colorView, depthView, w, h) (:104-112): torch CUDA float32
        [H,W,4] images."""
        for t in (color, depth):
            if tuple(t.shape) != (height, width, 4):
                raise ValueError(f"target shape {tuple(t.shape)} does not match {height}x{width}x4")
        self._target = (color, depth, int(width), int(height))

    def dispatch(self, clear: bool = False):
        """dispatch(encoder, clear) (:114-137): clear = attachments cleared to
        colour (0.05, 0.05, 0.05, 1) and depth 1 first (the pass the viewer
        draws, GpuRunner.svelte.ts:706); otherwise the splats are blended over
        the images' current contents."""
        if self._target is None:
            raise _lib.NpsError(-6, "splat forward dispatch: no target (set_target first)")
        color, depth, w, h = self._target
        self._opt.render(self._vp, w, h, color, depth, load=not clear)

    writeVPMatrix = write_vp_matrix
    setTarget = set_target
