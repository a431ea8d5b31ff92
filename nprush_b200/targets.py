"""Target preprocessing passes over libnprush_cuda (device images).

    blur(src, dst, direction=(1, 0), radius=8, sigma=4.0, flags=0)   <-> GpuBlurPipelineManager
    depth_aware_blur(color, depth, dst, radius=4)                     <-> GpuDepthAwareBlurPipelineManager
    splat_edge(depth, dst, thr_min=0.02, thr_max=0.06)               <-> the splat edge pass

Images are torch CUDA float32 tensors [H, W, 4] (depth in channel 0).  With
quantize=True the outputs hold what the reference's rgba8unorm textures hold.
"""
from __future__ import annotations

from . import _lib
from ._lib import call

SRGB_IN, SRGB_OUT = 1, 2


def _check(*ts):
    import torch
    for t in ts:
        assert isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
        assert t.ndim == 3 and t.shape[2] == 4
    torch.cuda.current_stream(ts[0].device).synchronize()


def blur(src, dst, direction=(1, 0), radius: int = 8, sigma: float = 4.0, flags: int = 0, quantize: bool = False):
    _check(src, dst)
    ctx = _lib.context(src.device.index or 0)
    call("nps_blur", ctx, src.data_ptr(), dst.data_ptr(), src.shape[1], src.shape[0], int(direction[0]),
         int(direction[1]), int(radius), int(flags), float(sigma), int(bool(quantize)))
    call("nps_sync", ctx)


def depth_aware_blur(color, depth, dst, radius: int = 4, quantize: bool = False):
    _check(color, depth, dst)
    ctx = _lib.context(color.device.index or 0)
    call("nps_depth_aware_blur", ctx, color.data_ptr(), depth.data_ptr(), dst.data_ptr(), color.shape[1],
         color.shape[0], int(radius), int(bool(quantize)))
    call("nps_sync", ctx)


def splat_edge(depth, dst, thr_min: float = 0.02, thr_max: float = 0.06, quantize: bool = False):
    _check(depth, dst)
    ctx = _lib.context(depth.device.index or 0)
    call("nps_splat_edge", ctx, depth.data_ptr(), dst.data_ptr(), depth.shape[1], depth.shape[0], float(thr_min),
         float(thr_max), int(bool(quantize)))
    call("nps_sync", ctx)
