"""Layered stroke fitting: splats, then three Bezier layers, one frame at a
time, as the reference's viewer loop orchestrates its managers
(src/lib/viewer/GpuRunner.svelte.ts:680-760, layer settings :262-280):

  1. the Sobel edge of the target depth (splat edge pass) and a depth-aware
     blur of the target colour are computed once per target;
  2. the splats fit the target (reference-semantics optimiser) and are rendered
     at the optimisation resolution;
  3. the edge layer (mode 0) fits the edge image;
  4. the base-colour layer (mode 1, no kill, kill thresholds 1e-4, ADC every
     150 dispatches, no background penalty) fits the blurred target over the
     splat render, and is then rendered over it;
  5. the fine colour layer (mode 1, max width 0.012, no kill, kill thresholds
     1e-4) fits the sharp target over splats + base layer.

All images are torch CUDA float tensors [H, W, 4] (depth [H, W]).
"""
from __future__ import annotations

import numpy as np


def mesh_targets(mesh, eye, center, width, height, fovy, up=(0.0, 0.0, 1.0), env=None, matcap=None,
                 path_trace_frames=0, shading_mode="normals"):
    """A frame's targets rendered from a mesh as the reference's viewer makes
    them (GpuRunner.svelte.ts:611-641): the mesh pass gives the colour target
    (normals or matcap shading) and the reciprocal-encoded depth; with
    path_trace_frames > 0 the path tracer's resolved output (that many samples
    per pixel) replaces the colour target, as the runner prefers it.  The
    Bezier layers' normal texture is the mesh pass's colour
    (GpuRunner.svelte.ts:400-430).  All three are rounded to 8 bits like the
    reference's render targets.

    Returns (target_rgba [H, W, 4], target_depth [H, W], normal_rgba [H, W, 4],
    vp, vp_inv) — torch CUDA tensors and the camera's column-major matrices."""
    from . import camera
    from .mesh_render import MeshRenderer
    from .path_trace import PathTracer
    vp, vpi = camera.view_proj(eye, center, fovy, width / height, up=up)
    view = camera.col_major(camera.look_at(eye, center, up))
    r = MeshRenderer(mesh, matcap=matcap, env=env)
    r.write_view_proj_mat(vp)
    r.write_view_mat(view)
    r.write_inv_view_proj_mat(vpi)
    r.write_shading_mode(shading_mode)
    color, depth4 = r.render(width, height, quantize=True)
    r.close()
    target = color
    if path_trace_frames > 0:
        pt = PathTracer(env_texture=env)
        pt.set_meshes(mesh)
        pt.set_output_size(width, height)
        pt.write_inv_view_proj_mat(vpi)
        pt.dispatch(frames=int(path_trace_frames), quantize=True)
        target = pt.output.clone()
        pt.close()
    return target, depth4[..., 0].contiguous(), color, vp, vpi


class LayeredFit:
    def __init__(self, target_rgba, target_depth, normal_rgba, vp, vp_inv, num_splats=512, num_beziers=256,
                 blur_radius=4, seed=0, layers=("edge", "base", "color")):
        import torch

        from . import targets
        from .bezier import GpuBezierOptimizerManager
        from .splat import GpuSplatOptimizerManager
        self.h, self.w = target_rgba.shape[0], target_rgba.shape[1]
        self.vp = np.ascontiguousarray(vp, np.float32).reshape(16)
        self.vpi = np.ascontiguousarray(vp_inv, np.float32).reshape(16)
        dev = target_rgba.device
        self.target = target_rgba.contiguous()
        self.depth = target_depth.contiguous()
        self.normal = normal_rgba.contiguous()
        depth4 = torch.zeros((self.h, self.w, 4), device=dev)
        depth4[..., 0] = self.depth
        # 1. per-target preprocessing, stored as the reference's rgba8unorm textures
        self.edge = torch.zeros_like(depth4)
        targets.splat_edge(depth4, self.edge, quantize=True)
        self.blurred = torch.zeros_like(self.target)
        targets.depth_aware_blur(self.target, depth4, self.blurred, blur_radius, quantize=True)
        self.zeros = torch.zeros_like(self.target)
        self.ones = torch.ones_like(self.depth)
        self.layers = tuple(layers)
        self.splats = GpuSplatOptimizerManager(num_splats, seed=seed)
        self.splats.write_splat_vp_matrix(self.vp, self.vpi)
        self.splats.set_backward_target(self.target, self.depth, self.w, self.h, borrow=True)
        self.splat_rgba = torch.zeros_like(self.target)
        self.splat_depth4 = torch.zeros_like(self.target)
        self.bg_after_base = torch.zeros_like(self.target)
        self.bz = {}
        for k, name in enumerate(self.layers):
            m = GpuBezierOptimizerManager(num_beziers, seed=seed + 1 + k)
            m.write_vp(self.vp, self.vpi)
            if name == "edge":
                m.write_mode(0.0)
                m.set_backward_target(self.edge, self.depth, self.zeros, self.ones, self.normal, self.w, self.h,
                                      borrow=True)
            elif name == "base":
                m.write_mode(1.0)
                m.write_bg_penalty(0.0)
                m.write_no_kill(True)
                m.write_kill_thresholds(0.0001, 0.0001)
                m.set_adc_period(150)
            elif name == "color":
                m.write_mode(1.0)
                m.write_max_width(0.012)
                m.write_kill_thresholds(0.0001, 0.0001)
                m.write_no_kill(True)
                m.write_bg_penalty(0.0)
            else:
                raise ValueError(name)
            self.bz[name] = m

    def frame(self):
        """One frame of training: splats, edge layer, base layer, colour layer."""
        self.splats.dispatch()
        self.splats.render(self.vp, self.w, self.h, self.splat_rgba, self.splat_depth4)
        splat_depth = self.splat_depth4[..., 0].contiguous()
        if "edge" in self.bz:
            self.bz["edge"].dispatch()
        bg = self.splat_rgba
        if "base" in self.bz:
            base = self.bz["base"]
            base.set_backward_target(self.blurred, self.depth, self.splat_rgba, splat_depth, self.normal, self.w,
                                     self.h)
            base.dispatch()
            # the base layer drawn over the splats is the next layer's background
            base.render(self.vp, self.w, self.h, self.bg_after_base, background=self.splat_rgba)
            bg = self.bg_after_base
        if "color" in self.bz:
            col = self.bz["color"]
            col.set_backward_target(self.target, self.depth, bg, splat_depth, self.normal, self.w, self.h)
            col.dispatch()
        self.last_background = bg

    def composite(self):
        """The finished picture: the colour layer over splats + base layer."""
        import torch
        out = torch.zeros_like(self.target)
        bg = self.bg_after_base if "base" in self.bz else self.splat_rgba
        if "color" in self.bz:
            self.bz["color"].render(self.vp, self.w, self.h, out, background=bg)
        else:
            out.copy_(bg)
        return out

    def close(self):
        self.splats.close()
        for m in self.bz.values():
            m.close()
