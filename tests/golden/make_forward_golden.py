"""Generates tests/golden/forward.npz: the display forwards drawn as their
render pipelines draw them.  The vertex and fragment stages are the
reference's own functions (src/lib/gpu/splat_forward.wgsl vert / frag,
src/lib/gpu/bezier_forward.wgsl vs_main / fs_main, translated to C++ by
oracle/build_ref.py with the instance counts baked in as their managers bake
them); the fixed-function steps between them are the restatement in
oracle/forward_raster.py.  Needs the reference checkout (NPRUSH_REFERENCE,
else oracle/reference_path.txt); the tests read only the .npz.

Cases (48 x 40 pixels):
* splats: 46 seeded splats of random shape, plus one of view depth 110 (past
  the camera's far plane at 100: the pipeline clips it away), one of view
  depth 99 (drawn) and one behind the camera (culled by the vertex stage);
  drawn on cleared attachments, and again over random contents (load);
* Bezier curves: 23 seeded curves plus one with a control point behind the
  camera (culled), with a random single-channel brush; cleared and over
  random contents.

    python tests/golden/make_forward_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))

import forward_raster as fr  # noqa: E402
from build_ref import RefModule  # noqa: E402
from scenes import bezier_scene, camera, splat_scene  # noqa: E402

W, H = 48, 40


def uniforms(vp):
    # ForwardUniforms {vp: mat4x4f, dims: vec2f, _pad: vec2f} (splat_forward.wgsl:15-19)
    return np.concatenate([np.asarray(vp, np.float32).reshape(16), np.array([W, H, 0, 0], np.float32)])


def splat_case():
    eye = (0.3, 0.4, 1.6)
    vp, _ = camera(W, H)
    s = splat_scene(49, 21, random_shape=True)
    e = np.array(eye, np.float64)
    fwd = -e / np.linalg.norm(e)  # the camera looks at the origin
    for k, depth in ((0, 110.0), (1, 99.0)):
        s[k, 0:3] = e + fwd * depth
        s[k, 3] = s[k, 12] = s[k, 15] = 6.0  # large enough to cover pixels at that distance
        s[k, 7] = 0.9
        s[k, 8:12] = (1.0, 0.0, 0.0, 0.0)
        s[k, 13], s[k, 14] = 2.0, 0.5
    s[2, 0:3] = e - fwd * 0.5  # behind the camera
    s[2, 7] = 0.9
    return s, vp


def draw_splats(s, vp, rgba, depth):
    m = RefModule("splat_forward", s.shape[0])
    m.bind(0, np.ascontiguousarray(s, np.float32))
    m.bind(1, uniforms(vp))

    def vert(vi, ii):
        return m.call("vert", np.array([vi, ii], np.uint32))

    def frag(fin):
        r = m.call("frag", fin)
        return None if m.discarded() else (r[0:4], r[4:8])

    # VsOut: pos 0-3, d 4-5, instance_idx 6 (flat), depth 7, conic 8-10 (flat)
    fr.draw(s.shape[0], 6, "triangle-list", vert, frag, W, H, [rgba, depth],
            [fr.blend_src_alpha, fr.blend_src_alpha], interp=[4, 5, 7], flat=[6, 8, 9, 10])


def bezier_case():
    vp, _ = camera(W, H, dist=1.4)
    b = bezier_scene(24, 22)
    b[0, 0:3] = np.array((0.3, 0.4, 1.4)) * 1.5  # p0 behind the camera (eye at (0.3, 0.4, 1.4))
    brush = np.random.default_rng(23).random((16, 32)).astype(np.float32)
    return b, vp, brush


def draw_beziers(b, vp, brush, rgba):
    m = RefModule("bezier_forward", b.shape[0])
    m.bind(0, np.ascontiguousarray(b, np.float32))
    m.bind(1, uniforms(vp))
    m.bind_sampler(2, True, "repeat", "clamp-to-edge")  # GpuBezierForwardPipelineManager.ts:34-41
    tex = np.zeros(brush.shape + (4,), np.float32)
    tex[..., 0] = brush
    m.bind_tex(3, tex)

    def vert(vi, ii):
        return m.call("vs_main", np.array([ii, vi], np.uint32))  # (instance_index, vertex_index)

    def frag(fin):
        r = m.call("fs_main", fin)
        return None if m.discarded() else (r[0:4],)

    # VsOut: pos 0-3, bezier_idx 4 (flat), p_screen 5-6
    fr.draw(b.shape[0], 4, "triangle-strip", vert, frag, W, H, [rgba], [fr.blend_premultiplied],
            interp=[5, 6], flat=[4])


def main():
    out = {}
    s, vp = splat_case()
    c = np.tile(np.array([0.05, 0.05, 0.05, 1.0], np.float32), (H, W, 1))  # the pass's clear values
    d = np.ones((H, W, 4), np.float32)
    draw_splats(s, vp, c, d)
    rng = np.random.default_rng(24)
    bc = rng.random((H, W, 4)).astype(np.float32)
    bd = rng.random((H, W, 4)).astype(np.float32)
    lc, ld = bc.copy(), bd.copy()
    draw_splats(s, vp, lc, ld)
    out.update(splat_params=s, splat_vp=np.asarray(vp, np.float32), splat_clear_rgba=c, splat_clear_depth=d,
               splat_bg_rgba=bc, splat_bg_depth=bd, splat_load_rgba=lc, splat_load_depth=ld)

    b, bvp, brush = bezier_case()
    cl = np.zeros((H, W, 4), np.float32)
    draw_beziers(b, bvp, brush, cl)
    bb = rng.random((H, W, 4)).astype(np.float32)
    bb[..., :3] *= bb[..., 3:4]  # premultiplied contents
    lb = bb.copy()
    draw_beziers(b, bvp, brush, lb)
    out.update(bezier_params=b, bezier_vp=np.asarray(bvp, np.float32), brush=brush, bezier_clear=cl,
               bezier_bg=bb, bezier_load=lb)
    np.savez_compressed(HERE / "forward.npz", **out)
    print("wrote", HERE / "forward.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
