"""Mesh render pass over libnprush_cuda — the host side of
GpuMeshRenderPipelineManager (src/lib/gpu/GpuMeshRenderPipelineManager.ts),
GpuEnvmapPipelineManager and the shared uniforms they read
(GpuUniformsBufferManager.ts), drawn as the viewer's optimisation pass draws
them (GpuRunner.svelte.ts:611-634).

    r = MeshRenderer(mesh, matcap=..., env=...)    # constructor({mesh}), matcap / env textures
    r.set_ground_mesh(ground)                       # setGroundMesh: drawn after the mesh
    r.set_pbr_mesh(mesh, albedo, normal_map)        # setPbrMesh: drawn last with the PBR stage
    r.write_view_proj_mat(vp); r.write_view_mat(v); r.write_inv_view_proj_mat(vpi)
    r.write_shading_mode("normals" | "shaded")
    color, depth = r.render(w, h)                   # envmap draw + addDraw into colour / depth targets

Images are torch CUDA float32 (h, w, 4) tensors; with quantize=True they hold
the 8-bit levels of the reference's render targets.  `depth` is the
reciprocal view-depth encoding 1 - 0.1 / max(w, 0.1) (1 where no triangle).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call
from .meshes import MeshData, concat


class MeshRenderer:
    def __init__(self, mesh: MeshData, matcap=None, env=None, device: int = 0):
        self.device = device
        self.ctx = _lib.context(device)
        self._h = ctypes.c_void_p()
        self.mesh, self.ground, self.pbr = mesh, None, None
        self.matcap = None if matcap is None else np.ascontiguousarray(matcap, np.float32)
        self.env = None if env is None else np.ascontiguousarray(env, np.float32)
        self.uniforms = np.zeros(52, np.float32)  # GpuUniformsBufferManager: 208 bytes
        self._rebuild()

    def _rebuild(self):
        parts = [self.mesh] + ([self.ground] if self.ground is not None else [])
        first_pbr = sum(p.n_tris for p in parts)
        if self.pbr is not None:
            parts.append(self.pbr[0])
        m = concat(parts)
        v = np.ascontiguousarray(m.vertices, np.float32)
        idx = np.ascontiguousarray(m.indices, np.uint32)
        self._destroy()
        call("nps_mesh_create", self.ctx, v.ctypes.data, v.shape[0], idx.ctypes.data if idx.size else None,
             idx.size // 3, ctypes.byref(self._h))
        if self.matcap is not None:
            self.set_matcap(self.matcap)
        if self.env is not None:
            self.set_env(self.env)
        if self.pbr is not None:
            _, alb, nm, srgb = self.pbr
            call("nps_mesh_set_pbr", self._h, first_pbr, alb.ctypes.data, alb.shape[1], alb.shape[0], int(bool(srgb)),
                 nm.ctypes.data, nm.shape[1], nm.shape[0])

    def set_ground_mesh(self, mesh: MeshData):
        self.ground = mesh
        self._rebuild()

    def set_pbr_mesh(self, mesh: MeshData, albedo, normal_map, srgb: bool = True):
        """The PBR-shaded mesh (the reference's textured ground), drawn last:
        albedo (sRGB-encoded unless srgb=False) and tangent-space normal map,
        (h, w, 4) float arrays."""
        self.pbr = (mesh, np.ascontiguousarray(albedo, np.float32), np.ascontiguousarray(normal_map, np.float32),
                    bool(srgb))
        self._rebuild()

    def set_matcap(self, rgba):
        self.matcap = np.ascontiguousarray(rgba, np.float32)
        call("nps_mesh_set_matcap", self._h, self.matcap.ctypes.data, self.matcap.shape[1], self.matcap.shape[0])

    def set_env(self, rgba):
        self.env = np.ascontiguousarray(rgba, np.float32)
        call("nps_mesh_set_env", self._h, self.env.ctypes.data, self.env.shape[1], self.env.shape[0])

    # GpuUniformsBufferManager's writers
    def write_view_proj_mat(self, m):
        self.uniforms[0:16] = np.asarray(m, np.float32).reshape(16)

    def write_view_mat(self, m):
        self.uniforms[16:32] = np.asarray(m, np.float32).reshape(16)

    def write_shading_mode(self, mode: str):
        if mode not in ("normals", "shaded"):  # the reference's parameter type
            raise ValueError(f"shading mode {mode!r}: 'normals' or 'shaded'")
        self.uniforms[32] = 0.0 if mode == "normals" else 1.0

    def write_inv_view_proj_mat(self, m):
        self.uniforms[36:52] = np.asarray(m, np.float32).reshape(16)

    def render(self, width: int, height: int, draw_env: bool = True, quantize: bool = True, out=None):
        """(colour, depth) of one pass; `out` may give the two tensors to fill."""
        import torch
        dev = f"cuda:{self.device}"
        if out is None:
            out = (torch.empty((height, width, 4), dtype=torch.float32, device=dev),
                   torch.empty((height, width, 4), dtype=torch.float32, device=dev))
        torch.cuda.current_stream(dev).synchronize()
        color, depth = out
        call("nps_mesh_render", self._h, self.uniforms.ctypes.data, color.data_ptr(), depth.data_ptr(), width, height,
             int(bool(draw_env)), int(bool(quantize)))
        call("nps_sync", self.ctx)
        return color, depth

    def _destroy(self):
        if self._h.value:
            call("nps_mesh_destroy", self._h)
            self._h = ctypes.c_void_p()

    def close(self):
        self._destroy()

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    # camelCase aliases (the reference's method names)
    setGroundMesh = set_ground_mesh
    setPbrMesh = set_pbr_mesh
    writeViewProjMat = write_view_proj_mat
    writeViewMat = write_view_mat
    writeShadingMode = write_shading_mode
    writeInvViewProjMat = write_inv_view_proj_mat


GpuMeshRenderPipelineManager = MeshRenderer
