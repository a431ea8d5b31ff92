"""Drives the reference's own compute shaders (compiled into oracle/_ref by
oracle/build_ref.py) with the buffer layouts the reference's managers create.

TEST INFRASTRUCTURE ONLY.  Buffer layouts follow
  GpuSplatOptimizerManager.ts:88-125   splats N*16 f32, grads N*16 i32,
                                       adam 2*16N f32 + t + pad, adc N f32,
                                       uniforms 160 B (vp, vp_inv, blur, pad)
  GpuBezierOptimizerManager.ts:97-136  beziers N*20 f32, grads N*18 i32,
                                       adam 2*18N + t, pixel_count, no_kill, pad,
                                       adc 2N f32, uniforms 160 B, pixel_loss 512^2 i32
and dispatch shapes follow the managers' dispatch() methods
(GpuSplatOptimizerManager.ts:365-388, GpuBezierOptimizerManager.ts:370-406).
"""
from __future__ import annotations

import numpy as np

from build_ref import REF_OUT, RefModule, reference_available

_cache: dict = {}


def mod(shader: str, n: int) -> RefModule:
    key = (shader, n)
    if key not in _cache:
        _cache[key] = RefModule(shader, n)
    return _cache[key]


def _tex(rgba):
    return np.ascontiguousarray(rgba, np.float32)


def _depth_tex(depth):
    d = np.zeros(depth.shape + (4,), np.float32)
    d[..., 0] = depth
    return d


def splat_backward(splats, vp, vpinv, tgt_rgba, tgt_depth):
    n = splats.shape[0]
    h, w = tgt_depth.shape
    m = mod("splat_backward", n)
    s = np.ascontiguousarray(splats, np.float32).copy()
    grads = np.zeros(n * 16, np.int32)
    uni = np.zeros(40, np.float32)
    uni[0:16] = vp
    uni[16:32] = vpinv
    m.bind(0, s)
    m.bind(1, grads)
    m.bind_tex(2, _tex(tgt_rgba))
    m.bind_tex(3, _depth_tex(tgt_depth))
    m.bind(4, uni)
    m.dispatch((w + 15) // 16, (h + 15) // 16, 1)
    return grads.reshape(n, 16)


def splat_step(splats, grads, m_, v_, adam_t, grad_accum):
    """Runs splat_step.wgsl; every workgroup reads the same adam.t (see below)."""
    n = splats.shape[0]
    md = mod("splat_step", n)
    s = np.ascontiguousarray(splats, np.float32).copy()
    g = np.ascontiguousarray(grads, np.int32).reshape(-1).copy()
    adam = np.zeros(32 * n + 8, np.float32)
    adam[0:16 * n] = m_.reshape(-1)
    adam[16 * n:32 * n] = v_.reshape(-1)
    adc = np.ascontiguousarray(grad_accum, np.float32).copy()
    md.bind(0, s)
    md.bind(1, g)
    md.bind(2, adam)
    md.bind(3, adc)
    gx = (n + 63) // 64
    # The shader lets invocation 0 write adam.t = t + 1 after a workgroup
    # barrier while every other workgroup reads adam.t: a cross-workgroup race.
    # The runner resolves it the way the shader intends (all read the old t).
    for x in range(gx):
        adam[32 * n] = adam_t
        md.run_one(x, 0, 0, gx, 1, 1)
    adam[32 * n] = adam_t + 1.0
    return s, g.reshape(n, 16), adam[:16 * n].reshape(n, 16), adam[16 * n:32 * n].reshape(n, 16), adc, adam_t + 1.0


def splat_adc(splats, m_, v_, adam_t, grad_accum):
    n = splats.shape[0]
    md = mod("splat_adc", n)
    s = np.ascontiguousarray(splats, np.float32).copy()
    adam = np.zeros(32 * n + 8, np.float32)
    adam[0:16 * n] = m_.reshape(-1)
    adam[16 * n:32 * n] = v_.reshape(-1)
    adam[32 * n] = adam_t
    adc = np.ascontiguousarray(grad_accum, np.float32).copy()
    md.bind(0, s)
    md.bind(1, adam)
    md.bind(2, adc)
    md.dispatch(1, 1, 1)
    return s, adam[:16 * n].reshape(n, 16), adam[16 * n:32 * n].reshape(n, 16), adc


def bezier_uniforms(vp, vpinv, mode=1.0, max_width=0.0, prune_alpha=0.0, prune_width=0.0, bg_penalty=0.0):
    uni = np.zeros(40, np.float32)
    uni[0:16] = vp
    uni[16:21] = [mode, max_width, prune_alpha, prune_width, bg_penalty]
    uni[24:40] = vpinv
    return uni


def bezier_backward(beziers, uni40, tgt_rgba, tgt_depth, bg_rgba, bg_depth, normal_rgba, adc=None, pixel_loss=None):
    n = beziers.shape[0]
    h, w = tgt_depth.shape
    md = mod("bezier_backward", n)
    b = np.ascontiguousarray(beziers, np.float32).copy()
    grads = np.zeros(n * 18, np.int32)
    adc = np.zeros(2 * n, np.float32) if adc is None else np.ascontiguousarray(adc, np.float32).copy()
    pl = np.zeros(512 * 512, np.int32) if pixel_loss is None else np.ascontiguousarray(pixel_loss, np.int32).copy()
    uni = np.ascontiguousarray(uni40, np.float32).copy()
    md.bind(0, b)
    md.bind(1, grads)
    md.bind_tex(2, _tex(tgt_rgba))
    md.bind_tex(3, _depth_tex(tgt_depth))
    md.bind(4, uni)
    md.bind_tex(5, _tex(bg_rgba))
    md.bind_tex(6, _depth_tex(bg_depth))
    md.bind(7, adc)
    md.bind_tex(8, _tex(normal_rgba))
    md.bind(9, pl)
    md.dispatch((w + 15) // 16, (h + 15) // 16, 1)
    return grads.reshape(n, 18), adc, pl


def bezier_step(beziers, grads, m_, v_, adam_t, pixel_count, no_kill, grad_accum, uni40):
    n = beziers.shape[0]
    md = mod("bezier_step", n)
    b = np.ascontiguousarray(beziers, np.float32).copy()
    g = np.ascontiguousarray(grads, np.int32).reshape(-1).copy()
    adam = np.zeros(36 * n + 8, np.float32)
    adam[0:18 * n] = m_.reshape(-1)
    adam[18 * n:36 * n] = v_.reshape(-1)
    adam[36 * n + 1] = pixel_count
    adam[36 * n + 2] = no_kill
    adc = np.zeros(2 * n, np.float32)
    adc[:n] = grad_accum
    uni = np.ascontiguousarray(uni40, np.float32).copy()
    md.bind(0, b)
    md.bind(1, g)
    md.bind(2, adam)
    md.bind(3, adc)
    md.bind(4, uni)
    gx = (n + 63) // 64
    for x in range(gx):  # same adam.t resolution as splat_step
        adam[36 * n] = adam_t
        md.run_one(x, 0, 0, gx, 1, 1)
    return b, g.reshape(n, 18), adam[:18 * n].reshape(n, 18), adam[18 * n:36 * n].reshape(n, 18), adc[:n], adam_t + 1.0


def bezier_adc(beziers, m_, v_, adam_t, no_kill, grad_accum, loss_accum, pixel_loss, uni40):
    n = beziers.shape[0]
    md = mod("bezier_adc", n)
    b = np.ascontiguousarray(beziers, np.float32).copy()
    adam = np.zeros(36 * n + 8, np.float32)
    adam[0:18 * n] = m_.reshape(-1)
    adam[18 * n:36 * n] = v_.reshape(-1)
    adam[36 * n] = adam_t
    adam[36 * n + 2] = no_kill
    adc = np.zeros(2 * n, np.float32)
    adc[:n] = grad_accum
    adc[n:] = loss_accum
    pl = np.ascontiguousarray(pixel_loss, np.int32).copy()
    uni = np.ascontiguousarray(uni40, np.float32).copy()
    md.bind(0, b)
    md.bind(1, adam)
    md.bind(2, adc)
    md.bind(3, pl)
    md.bind(4, uni)
    md.dispatch(1, 1, 1)
    return b, adam[:18 * n].reshape(n, 18), adam[18 * n:36 * n].reshape(n, 18), adc[:n], adc[n:], pl


def build_bvh(vertices, indices):
    """The reference's own buildBvh (bvh.ts:202-223, translated by
    oracle/ts2py.py) on MeshData-layout vertices (V x 12 f32) and triangle
    indices: (nodes (N, 8) float32 holding the u32 fields' bits in columns 3
    and 7, tri_indices (T, 3) uint32), the layout of oracle/bvh.py."""
    import js_rt
    from build_ref import load_ts
    if "bvh" not in _cache:
        _cache["bvh"] = load_ts("bvh")
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    r = _cache["bvh"].buildBvh(js_rt.Float32Array(v.tolist()), js_rt.Uint32Array(i.tolist()))
    nodes = np.frombuffer(bytes(r.nodes.b), np.float32).reshape(-1, 8).copy()
    return nodes, r.triIndices.a.reshape(-1, 3).copy()


def stage_module(shader: str) -> RefModule:
    """A render pipeline's translated stages: built from the reference checkout
    when present, else the build already under oracle/_ref."""
    if reference_available():
        return RefModule(shader, 0)
    found = sorted(REF_OUT.glob(f"{shader}_n0_*.so"))
    if not found:
        raise FileNotFoundError(f"oracle/_ref has no {shader} build and the reference checkout is absent")
    return RefModule.from_path(found[-1])


class MeshStages:
    """mesh.wgsl vert / frag / frag_pbr and envmap.wgsl frag, the reference's
    own functions, with the bindings the managers create (uniforms at 0,
    matcap + clamped linear sampler at 1-2, the PBR textures + repeating
    sampler at 3-5, GpuMeshRenderPipelineManager.ts:226-246; environment +
    u-repeating sampler, GpuEnvmapPipelineManager.ts): the stage interface
    that oracle/mesh_raster.render drives."""

    def __init__(self, uni, matcap, env, albedo=None, normal_map=None):
        self.mesh = stage_module("mesh")
        self.envm = stage_module("envmap")
        self.uni = np.ascontiguousarray(uni, np.float32)
        for m in (self.mesh, self.envm):
            m.bind(0, self.uni)
        self.mesh.bind_tex(1, np.ascontiguousarray(matcap, np.float32))
        self.mesh.bind_sampler(2, True, "clamp-to-edge", "clamp-to-edge")
        if albedo is not None:
            self.mesh.bind_tex(3, np.ascontiguousarray(albedo, np.float32))
            self.mesh.bind_tex(4, np.ascontiguousarray(normal_map, np.float32))
            self.mesh.bind_sampler(5, True, "repeat", "repeat")
        self.envm.bind_tex(1, np.ascontiguousarray(env, np.float32))
        self.envm.bind_sampler(2, True, "repeat", "clamp-to-edge")

    def vert(self, vin, uni):
        return self.mesh.call("vert", np.asarray(vin, np.float32))

    def frag(self, vo, uni, pbr=False):
        r = self.mesh.call("frag_pbr" if pbr else "frag", np.asarray(vo, np.float32))
        return r[0:4], r[4:8]

    def env_frag(self, ndc, uni):
        return self.envm.call("frag", np.array([0, 0, 0, 1, ndc[0], ndc[1]], np.float32))


def path_trace(vertices, nodes, tri_indices, env_rgba, inv_view_proj, frame, accum):
    """One dispatch of path_trace.wgsl (GpuPathTracePipelineManager.ts:222-240):
    adds one sample per pixel to accum (h, w, 4) float32 in place.  Bindings
    as the manager creates them (:60-72, 196-210): uniforms 80 B
    [invViewProjMat, frame, num_tris, out_w, out_h], vertices, bvh nodes,
    bvh triangle indices, accum, env texture + linear sampler (u repeat, v
    clamp-to-edge)."""
    h, w = accum.shape[:2]
    m = mod("path_trace", 0)
    uni = np.zeros(20, np.uint32)
    uni[:16] = np.ascontiguousarray(inv_view_proj, np.float32).reshape(16).view(np.uint32)
    uni[16:20] = [frame, tri_indices.shape[0], w, h]
    m.bind(0, uni)
    m.bind(1, np.ascontiguousarray(vertices, np.float32).reshape(-1))
    m.bind(2, np.ascontiguousarray(nodes, np.float32).reshape(-1))
    m.bind(3, np.ascontiguousarray(tri_indices, np.uint32).reshape(-1))
    assert accum.dtype == np.float32 and accum.flags.c_contiguous
    m.bind(4, accum)
    m.bind_tex(5, _tex(env_rgba))
    m.bind_sampler(6, True, "repeat", "clamp-to-edge")
    m.dispatch(-(-w // 8), -(-h // 8))
    return accum


def path_trace_resolve(accum):
    """path_trace_resolve.wgsl: the stored floats of the rgba8unorm output."""
    h, w = accum.shape[:2]
    m = mod("path_trace_resolve", 0)
    out = np.zeros((h, w, 4), np.float32)
    uni = np.array([w, h, 0, 0], np.uint32)
    m.bind(0, np.ascontiguousarray(accum, np.float32))
    m.bind_storage_tex(1, out)
    m.bind(2, uni)
    m.dispatch(-(-w // 8), -(-h // 8))
    return out
