"""GPU mesh render pass (nps_mesh_*) against tests/golden/mesh_raster.npz
(the reference's own mesh.wgsl / envmap.wgsl stage functions between the
restated fixed-function steps) and the CPU restatement.

Tolerances: the kernels are compiled without FMA contraction and use the
restatement's exact integer edge functions, so coverage, depth test and
every covered pixel's colour and depth match exactly; background pixels go
through atan2f / asinf, whose last place can differ from the C library's,
and are compared at 2e-5."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLD = Path(__file__).resolve().parent / "golden" / "mesh_raster.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def mrmod():
    from nprush_b200 import build
    build.build()
    from nprush_b200 import mesh_render
    return mesh_render


def render(mrmod, verts, idx, uni, w, h, matcap, env, draw_env=True, quantize=False):
    from nprush_b200.meshes import MeshData
    r = mrmod.MeshRenderer(MeshData(np.asarray(verts, np.float32), np.asarray(idx, np.uint32)), matcap=matcap,
                           env=env)
    r.uniforms[:] = uni
    c, d = r.render(w, h, draw_env=draw_env, quantize=quantize)
    out = c.cpu().numpy(), d.cpu().numpy()
    r.close()
    return out


def check(got_c, got_d, want_c, want_d):
    covered = want_d[..., 0] < 1.0
    np.testing.assert_array_equal(got_d[..., 0] < 1.0, covered)
    np.testing.assert_array_equal(got_d, want_d)
    np.testing.assert_array_equal(got_c[covered], want_c[covered])
    np.testing.assert_allclose(got_c[~covered], want_c[~covered], atol=2e-5, rtol=0)


@pytest.mark.parametrize("mode", ["normals", "shaded"])
def test_matches_reference_fixture(mrmod, gold, mode):
    h, w = gold[f"color_{mode}"].shape[:2]
    c, d = render(mrmod, gold["vertices"], gold["indices"], gold[f"uniforms_{mode}"], w, h, gold["matcap"],
                  gold["env"])
    check(c, d, gold[f"color_{mode}"], gold[f"depth_{mode}"])
    # the 8-bit targets: the same levels except where the float sits on a rounding edge
    cq, dq = render(mrmod, gold["vertices"], gold["indices"], gold[f"uniforms_{mode}"], w, h, gold["matcap"],
                    gold["env"], quantize=True)
    for got, want in ((cq, gold[f"color_{mode}"]), (dq, gold[f"depth_{mode}"])):
        wq = np.rint(np.clip(want, 0, 1) * 255) / 255
        frac = np.clip(want, 0, 1) * 255 - np.floor(np.clip(want, 0, 1) * 255)
        assert np.all((np.abs(got - wq) < 1e-6) | (np.abs(frac - 0.5) < 1e-3))


@pytest.mark.parametrize("mode", ["normals", "shaded"])
def test_pbr_ground_matches_reference_fixture(mrmod, gold, mode):
    from nprush_b200.meshes import MeshData
    h, w = gold[f"pbr_color_{mode}"].shape[:2]
    first = int(gold["pbr_first"])
    v, idx = gold["pbr_vertices"], gold["pbr_indices"]
    # the scene split as the manager holds it: mesh, then the PBR mesh (linear albedo)
    r = mrmod.MeshRenderer(MeshData(v[:v.shape[0] - 4], idx[:3 * first]), matcap=gold["matcap"], env=gold["env"])
    r.set_pbr_mesh(MeshData(v[v.shape[0] - 4:], idx[3 * first:] - np.uint32(v.shape[0] - 4)), gold["albedo"],
                   gold["normal_map"], srgb=False)
    r.uniforms[:] = gold[f"uniforms_{mode}"]
    c, d = (t.cpu().numpy() for t in r.render(w, h, quantize=False))
    check(c, d, gold[f"pbr_color_{mode}"], gold[f"pbr_depth_{mode}"])
    # an sRGB-encoded albedo gives the linear one's image (decoded per texel)
    enc = gold["albedo"].copy()
    lin = enc[..., :3].astype(np.float64)
    enc[..., :3] = np.where(lin > 0.0031308, 1.055 * lin ** (1 / 2.4) - 0.055, lin * 12.92)
    r.set_pbr_mesh(r.pbr[0], enc, gold["normal_map"], srgb=True)
    r.uniforms[:] = gold[f"uniforms_{mode}"]
    c2, d2 = (t.cpu().numpy() for t in r.render(w, h, quantize=False))
    np.testing.assert_array_equal(d2, d)
    np.testing.assert_allclose(c2, c, atol=1e-5, rtol=0)
    r.close()


def _scene_uniforms(w, h, eye=(4.0, -3.5, 2.6), target=(0.0, 0.0, 0.3), mode=0.0):
    from nprush_b200 import camera
    vp, inv = camera.view_proj(eye, target, 0.9, w / h, up=(0.0, 0.0, 1.0))
    u = np.zeros(52, np.float32)
    u[0:16], u[16:32], u[32], u[36:52] = vp, camera.col_major(camera.look_at(eye, target, (0.0, 0.0, 1.0))), mode, inv
    return u


def test_larger_scene_against_restatement(mrmod):
    """~6k triangles at 96 x 72 against the full CPU restatement."""
    import mesh_raster as mr
    from nprush_b200 import meshes
    sc = meshes.demo_scene(12, seed=11, sphere_detail=12)
    w, h = 96, 72
    uni = _scene_uniforms(w, h, mode=1.0)
    matcap, env = np.random.default_rng(1).random((16, 16, 4)).astype(np.float32), meshes.sky_env(64, 32)
    c, d = render(mrmod, sc.vertices, sc.indices, uni, w, h, matcap, env)
    wc, wd = mr.render(sc.vertices, sc.indices, uni, w, h, mr.RestatedStages(matcap, env))
    check(c, d, wc, wd)


def test_draw_order_decides_equal_depths(mrmod):
    """Two coplanar quads: where they overlap the depths are equal and the one
    drawn first keeps the pixel (depth "less")."""
    import mesh_raster as mr
    from nprush_b200 import meshes
    a = meshes.quad((0.0, 0.0, 0.0), 2.0, (1.0, 0.0, 0.0, 1.0))
    b = meshes.quad((0.5, 0.3, 0.0), 2.0, (0.0, 0.0, 1.0, 1.0))
    b.vertices[:, 3:6] = (0.0, 0.6, 0.8)  # a different normal: a different colour in normals mode
    sc = meshes.concat([a, b])
    w, h = 48, 40
    uni = _scene_uniforms(w, h, eye=(0.3, -2.0, 2.5), target=(0.2, 0.1, 0.0))
    env = meshes.sky_env(32, 16)
    c, d = render(mrmod, sc.vertices, sc.indices, uni, w, h, np.ones((1, 1, 4), np.float32), env)
    wc, wd = mr.render(sc.vertices, sc.indices, uni, w, h, mr.RestatedStages(np.ones((1, 1, 4), np.float32), env))
    check(c, d, wc, wd)
    first = np.array([0.5, 0.5, 1.0]) * 4  # normal (0, 0, 1) -> colour before Reinhard
    assert (np.abs(c[..., 2] - first[2] / (first[2] + 1)) < 1e-6).sum() > 50


def test_background_and_empty_mesh(mrmod, gold):
    h, w = gold["color_normals"].shape[:2]
    c, d = render(mrmod, np.zeros((0, 12), np.float32), np.zeros(0, np.uint32), gold["uniforms_normals"], w, h,
                  gold["matcap"], gold["env"])
    assert np.all(d == 1.0)
    sky = gold["depth_normals"][..., 0] == 1.0
    np.testing.assert_allclose(c[sky], gold["color_normals"][sky], atol=2e-5, rtol=0)
    c, d = render(mrmod, gold["vertices"], gold["indices"], gold["uniforms_normals"], w, h, gold["matcap"],
                  gold["env"], draw_env=False)
    np.testing.assert_array_equal(c[sky], np.broadcast_to(np.float32([0.05, 0.05, 0.05, 1.0]), c[sky].shape))


def test_bad_arguments(mrmod):
    from nprush_b200 import _lib
    from nprush_b200.meshes import MeshData
    with pytest.raises(_lib.NpsError):
        mrmod.MeshRenderer(MeshData(np.zeros((3, 12), np.float32), np.array([0, 1, 3], np.uint32)))


def test_clipping_edge_cases_match_restatement(mrmod):
    """Behind the eye, guard-band and far-plane clipping, degenerate and
    offscreen triangles: the kernels draw exactly what the restatement does."""
    import mesh_raster as mr
    from nprush_b200 import camera
    w, h = 40, 30
    eye, tgt = (0.0, -3.0, 0.0), (0.0, 0.0, 0.0)
    vp, inv = camera.view_proj(eye, tgt, 0.9, w / h, up=(0.0, 0.0, 1.0))
    u = np.zeros(52, np.float32)
    u[0:16], u[36:52] = vp, inv
    u[16:32] = camera.col_major(camera.look_at(eye, tgt, (0.0, 0.0, 1.0)))
    tris = [((-1, -5, -1), (1, -5, -1), (0, -5, 1)),
            ((-1e4, 2.0, -1e4), (1e4, 2.0, -1e4), (0.0, 2.0, 1e4)),
            ((-0.5, 1.0, -0.5), (0.5, 1.0, -0.5), (0.0, 500.0, 0.3)),
            ((0, 1, 0), (0.5, 1, 0), (1, 1, 0)),
            ((50, 1, 0), (51, 1, 0), (50, 1, 1))]
    one = np.ones((1, 1, 4), np.float32)
    for t in tris:
        v = np.zeros((6, 12), np.float32)
        v[:3, 0:3] = t
        v[3:, 0:3] = t
        v[:, 5] = 1.0
        v[:, 6:10] = (0.5, 0.5, 0.5, 1.0)
        idx = np.array([0, 1, 2, 3, 5, 4], np.uint32)
        c, d = render(mrmod, v, idx, u, w, h, one, one)
        wc, wd = mr.render(v, idx, u, w, h, mr.RestatedStages(one, one))
        check(c, d, wc, wd)
