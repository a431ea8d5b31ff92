"""Target preprocessing passes over libnprush_cuda (device images).

    blur(src, dst, direction=(1, 0), radius=8, sigma=4.0, flags=0)   <-> one pass of blur.wgsl
    depth_aware_blur(color, depth, dst, radius=4)                     <-> depth_aware_blur.wgsl
    splat_edge(depth, dst, thr_min=0.02, thr_max=0.06)               <-> the splat edge pass

and the manager classes with the reference's call shape:

    GpuBlurPipelineManager().blur(src, dst, temp, w, h, radius, sigma, is_srgb)
    GpuDepthAwareBlurPipelineManager().blur(color, depth, dst, w, h, radius)

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


def _check_size(width, height, *ts):
    for t in ts:
        if (int(t.shape[1]), int(t.shape[0])) != (int(width), int(height)):
            raise ValueError(f"image {tuple(t.shape)} is not {width}x{height}")


class GpuBlurPipelineManager:
    """GpuBlurPipelineManager (src/lib/gpu/GpuBlurPipelineManager.ts:46-99):
    the separable Gaussian blur as the reference runs it, a horizontal pass
    src -> temp (sRGB decoded on input when is_srgb) and a vertical pass
    temp -> dst (sRGB encoded on output).  The viewer's temp and destination
    textures are rgba8unorm (GpuRunner.svelte.ts:359, :380-384), so both passes
    store 8-bit levels unless quantize=False."""

    def blur(self, src, dst, temp, width: int, height: int, radius: int, sigma: float, is_srgb: bool = False,
             quantize: bool = True):
        _check_size(width, height, src, dst, temp)
        blur(src, temp, (1, 0), radius, sigma, SRGB_IN if is_srgb else 0, quantize=quantize)
        blur(temp, dst, (0, 1), radius, sigma, SRGB_OUT if is_srgb else 0, quantize=quantize)


class GpuDepthAwareBlurPipelineManager:
    """GpuDepthAwareBlurPipelineManager (src/lib/gpu/GpuDepthAwareBlurPipelineManager.ts:41-70)."""

    def blur(self, color, depth, dst, width: int, height: int, radius: int, quantize: bool = True):
        _check_size(width, height, color, depth, dst)
        depth_aware_blur(color, depth, dst, radius, quantize=quantize)
