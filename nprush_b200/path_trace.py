"""Path-traced targets over libnprush_cuda — the host side of
GpuPathTracePipelineManager (src/lib/gpu/GpuPathTracePipelineManager.ts).

    pt = PathTracer(env_texture=sky)          # constructor({device, envTexture})
    pt.set_meshes([mesh, ground])             # setMeshes: concatenation + SAH BVH
    pt.set_output_size(w, h)                  # setOutputSize: accum + output images
    pt.write_inv_view_proj_mat(vp_inv)        # writeInvViewProjMat
    pt.reset()                                # reset: clear the accumulation
    pt.dispatch()                             # dispatch: one sample per pixel + resolve
    pt.output                                 # (h, w, 4) float32 CUDA tensor (the output texture)

`dispatch(frames=n)` adds n samples in one launch, equal to n dispatches.
Images are torch CUDA float32 tensors; `output` holds the rgba8unorm levels
the reference's output texture holds (quantize=False keeps the floats).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call
from .meshes import MeshData, concat


def build_bvh(vertices, indices):
    """buildBvh (bvh.ts:202-223) on the host: (nodes (N, 8) float32 with u32
    bits in columns 3 and 7, tri_indices (T, 3) uint32)."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 12)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    t = idx.shape[0] // 3
    nodes = np.zeros((max(1, 2 * t - 1), 8), np.float32)
    tris = np.zeros((max(1, t), 3), np.uint32)
    nn = ctypes.c_uint32()
    call("nps_bvh_build", v.ctypes.data, v.shape[0], idx.ctypes.data if t else None, t, nodes.ctypes.data,
         tris.ctypes.data, ctypes.byref(nn))
    return nodes[: nn.value].copy(), tris[:t].copy()


class PathTracer:
    def __init__(self, env_texture=None, device: int = 0):
        self.device = device
        self.ctx = _lib.context(device)
        self._h = ctypes.c_void_p()
        self.env = None if env_texture is None else np.ascontiguousarray(env_texture, np.float32)
        self.accum = None
        self.output = None
        self.width = self.height = 0
        self.frame_count = 0
        self.inv_view_proj = np.eye(4, dtype=np.float32).reshape(16)
        self.num_tris = 0

    # -- scene
    def set_meshes(self, meshes):
        m = meshes if isinstance(meshes, MeshData) else concat(
            [x if isinstance(x, MeshData) else MeshData(*x) for x in meshes])
        v = np.ascontiguousarray(m.vertices, np.float32)
        idx = np.ascontiguousarray(m.indices, np.uint32)
        self._destroy()
        call("nps_pt_create", self.ctx, v.ctypes.data, v.shape[0], idx.ctypes.data if idx.size else None,
             idx.size // 3, ctypes.byref(self._h))
        self.num_tris = idx.size // 3
        if self.env is not None:
            self.set_env(self.env)

    def set_env(self, rgba):
        rgba = np.ascontiguousarray(rgba, np.float32)
        assert rgba.ndim == 3 and rgba.shape[2] == 4
        self.env = rgba
        if self._h.value:
            call("nps_pt_set_env", self._h, rgba.ctypes.data, rgba.shape[1], rgba.shape[0])

    def bvh(self):
        """(nodes, tri_indices) of the uploaded BVH."""
        nn, nt = ctypes.c_uint32(), ctypes.c_uint32()
        call("nps_pt_bvh_size", self._h, ctypes.byref(nn), ctypes.byref(nt))
        nodes = np.zeros((nn.value, 8), np.float32)
        tris = np.zeros((max(1, nt.value), 3), np.uint32)
        call("nps_pt_read_bvh", self._h, nodes.ctypes.data, tris.ctypes.data)
        return nodes, tris[: nt.value]

    # -- images
    def set_output_size(self, width: int, height: int):
        if width == self.width and height == self.height and self.accum is not None:
            return
        import torch
        dev = f"cuda:{self.device}"
        self.accum = torch.zeros((height, width, 4), dtype=torch.float32, device=dev)
        self.output = torch.zeros((height, width, 4), dtype=torch.float32, device=dev)
        torch.cuda.current_stream(dev).synchronize()
        self.width, self.height = width, height
        self.frame_count = 0

    def reset(self):
        if self.accum is None:
            return
        import torch
        self.accum.zero_()
        torch.cuda.current_stream(self.accum.device).synchronize()
        self.frame_count = 0

    def write_inv_view_proj_mat(self, mat):
        self.inv_view_proj = np.ascontiguousarray(mat, np.float32).reshape(16)

    def trace(self, frames: int = 1):
        """The path-trace pass alone (asynchronous on the library's stream)."""
        m = self.inv_view_proj
        call("nps_pt_trace", self._h, m.ctypes.data, self.frame_count, int(frames), self.accum.data_ptr(),
             self.width, self.height)
        self.frame_count += int(frames)

    def dispatch(self, frames: int = 1, quantize: bool = True, sync: bool = True):
        if not self._h.value or self.accum is None:
            return
        self.trace(frames)
        call("nps_pt_resolve", self.ctx, self.accum.data_ptr(), self.output.data_ptr(), self.width, self.height,
             int(bool(quantize)))
        if sync:
            call("nps_sync", self.ctx)

    def overflows(self) -> int:
        c = ctypes.c_uint32()
        call("nps_pt_overflows", self._h, ctypes.byref(c))
        return c.value

    # -- lifetime
    def _destroy(self):
        if self._h.value:
            call("nps_pt_destroy", self._h)
            self._h = ctypes.c_void_p()

    def close(self):
        self._destroy()

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    # camelCase aliases (the reference's method names)
    setMeshes = set_meshes
    setOutputSize = set_output_size
    writeInvViewProjMat = write_inv_view_proj_mat


GpuPathTracePipelineManager = PathTracer
