"""Mesh render pass on the CPU: the restatement (oracle/mesh_raster.py)
against tests/golden/mesh_raster.npz, whose vertex and fragment stages are the
reference's own mesh.wgsl / envmap.wgsl functions run on the host, plus
properties of the fixed-function part (clipping, the fill rule, culling)."""
from pathlib import Path

import numpy as np
import pytest

import mesh_raster as mr
from conftest import requires_reference

GOLD = Path(__file__).resolve().parent / "golden" / "mesh_raster.npz"
F = np.float32


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("mode", ["normals", "shaded"])
def test_restatement_matches_fixture(gold, mode):
    h, w = gold[f"color_{mode}"].shape[:2]
    st = mr.RestatedStages(gold["matcap"], gold["env"])
    c, d = mr.render(gold["vertices"], gold["indices"], gold[f"uniforms_{mode}"], w, h, st)
    np.testing.assert_array_equal(c, gold[f"color_{mode}"])
    np.testing.assert_array_equal(d, gold[f"depth_{mode}"])


@pytest.mark.parametrize("mode", ["normals", "shaded"])
def test_restatement_matches_fixture_pbr(gold, mode):
    """The scene with a ground drawn last through the PBR stage (albedo and
    normal map repeating 3 x 3); the fixture ran the reference's frag_pbr."""
    h, w = gold[f"pbr_color_{mode}"].shape[:2]
    st = mr.RestatedStages(gold["matcap"], gold["env"], gold["albedo"], gold["normal_map"])
    c, d = mr.render(gold["pbr_vertices"], gold["pbr_indices"], gold[f"uniforms_{mode}"], w, h, st,
                     first_pbr=int(gold["pbr_first"]))
    np.testing.assert_array_equal(c, gold[f"pbr_color_{mode}"])
    np.testing.assert_array_equal(d, gold[f"pbr_depth_{mode}"])
    assert np.abs(c - gold[f"color_{mode}"]).max() > 0.05  # the textured ground shows


def test_fixture_sanity(gold):
    d = gold["depth_normals"][..., 0]
    assert 0.5 < (d < 1).mean() < 0.98      # geometry and sky both present
    c = gold["color_normals"]
    assert np.all((c >= 0) & (c <= 1))
    assert not np.array_equal(gold["color_normals"], gold["color_shaded"])
    np.testing.assert_array_equal(gold["depth_normals"], gold["depth_shaded"])


def test_clipping():
    one_hot = np.eye(3, dtype=np.float32)
    inside = [np.array([0, 0, 0.5, 1], np.float32), np.array([1, 0, 0.5, 1], np.float32),
              np.array([0, 1, 0.5, 1], np.float32)]
    assert len(mr.clip_polygon(inside, one_hot)) == 3
    behind = [p * np.array([1, 1, -1, 1], np.float32) for p in inside]
    assert mr.clip_polygon(behind, one_hot) == []
    straddle = [np.array([0, 0, -0.5, 1], np.float32), np.array([1, 0, 0.5, 1], np.float32),
                np.array([0, 1, 0.5, 1], np.float32)]
    poly = mr.clip_polygon(straddle, one_hot)
    assert len(poly) == 4
    for p, c in poly:
        assert p[2] >= 0 and p[3] - p[2] >= 0
        np.testing.assert_allclose(c.sum(), 1.0, atol=1e-6)   # weights of the original vertices


def test_shared_edges_cover_each_pixel_once():
    """Convex quads split into two triangles: every pixel centre strictly
    inside the quad is claimed by exactly one triangle, and none by two, also
    where centres lie exactly on the shared diagonal (the snapped, exact edge
    functions and the top-left rule)."""
    rng = np.random.default_rng(0)
    w = h = 24
    for trial in range(30):
        ang = np.sort(rng.uniform(0, 2 * np.pi, 4))[::-1]  # clockwise in y-down screen space
        rad = rng.uniform(4, 11, 2)
        cen = rng.uniform(9, 15, 2)
        c = np.round((cen + np.stack([np.cos(ang) * rad[0], np.sin(ang) * rad[1]], 1)) * 2) / 2
        clip = [np.array([x / w * 2 - 1, 1 - y / h * 2, 0.5, 1.0], np.float32) for x, y in c]
        count = np.zeros((h, w), np.int32)
        for tri in ((0, 1, 2), (0, 2, 3)):
            for order_ in (tri, tri[::-1]):
                poly = mr.clip_polygon([clip[i] for i in order_], np.eye(3, dtype=np.float32))
                st = mr.setup(poly, 0, w, h)
                if st is None:
                    continue
                bx0, bx1, by0, by1 = st["box"]
                py, px = np.mgrid[by0:by1 + 1, bx0:bx1 + 1]
                ins, _, _ = mr.coverage(st, px, py)
                count[by0:by1 + 1, bx0:bx1 + 1] += ins
        assert count.max() <= 1, f"trial {trial}: a pixel covered twice"
        # centres strictly inside the quad (exact test on the snapped corners)
        X, Y = np.rint(c[:, 0] * 256).astype(np.int64), np.rint(c[:, 1] * 256).astype(np.int64)
        py, px = np.mgrid[0:h, 0:w]
        cx, cy = px * 256 + 128, py * 256 + 128
        e = [(Y[(i + 1) % 4] - Y[i]) * (cx - X[i]) - (X[(i + 1) % 4] - X[i]) * (cy - Y[i]) for i in range(4)]
        strictly = np.all([ei < 0 for ei in e], 0) | np.all([ei > 0 for ei in e], 0)
        assert np.all(count[strictly] == 1), f"trial {trial}: a hole"


def test_back_faces_are_culled():
    from nprush_b200 import camera, meshes
    box = meshes.box((0.0, 0.0, 0.0), 0.5)
    vp, inv = camera.view_proj((2.0, 1.5, 1.2), (0.0, 0.0, 0.0), 0.9, 1.0, up=(0.0, 0.0, 1.0))
    uni = np.zeros(52, np.float32)
    uni[0:16], uni[36:52] = vp, inv
    uni[16:32] = camera.col_major(camera.look_at((2.0, 1.5, 1.2), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0)))
    st = mr.RestatedStages(np.ones((1, 1, 4), np.float32), np.ones((1, 1, 4), np.float32))
    front = [t for t in range(12) if any(
        mr.setup(mr.clip_polygon([mr.vert(box.vertices[i], uni)[0:4] for i in box.indices[3 * t:3 * t + 3]],
                                 np.eye(3, dtype=np.float32)), 0, 32, 32) is not None for _ in [0])]
    assert len(front) == 6   # three faces of the box face the camera
    c, d = mr.render(box.vertices, box.indices, uni, 32, 32, st)
    assert (d[..., 0] < 1).sum() > 100


@requires_reference
def test_reference_stages_reproduce_the_fixtures(tmp_path, monkeypatch):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", GOLD.parent / "make_mesh_raster_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    monkeypatch.setattr(mk, "HERE", tmp_path)
    mk.main()
    a, b = np.load(GOLD), np.load(tmp_path / "mesh_raster.npz")
    for k in a.files:
        np.testing.assert_array_equal(a[k], b[k])


def _uni(eye, target, w, h, fovy=0.9):
    from nprush_b200 import camera
    vp, inv = camera.view_proj(eye, target, fovy, w / h, up=(0.0, 0.0, 1.0))
    u = np.zeros(52, np.float32)
    u[0:16], u[36:52] = vp, inv
    u[16:32] = camera.col_major(camera.look_at(eye, target, (0.0, 0.0, 1.0)))
    return u


def _tri(p0, p1, p2):
    v = np.zeros((3, 12), np.float32)
    v[:, 0:3] = (p0, p1, p2)
    v[:, 5] = 1.0
    v[:, 6:10] = (0.5, 0.5, 0.5, 1.0)
    return v


def _both_windings(v):
    return np.concatenate([v, v]), np.array([0, 1, 2, 3, 5, 4], np.uint32)


def test_clipping_and_culling_edge_cases():
    w, h = 40, 30
    st = mr.RestatedStages(np.ones((1, 1, 4), np.float32), np.ones((1, 1, 4), np.float32))
    uni = _uni((0.0, -3.0, 0.0), (0.0, 0.0, 0.0), w, h)  # looking along +y
    # behind the eye: nothing drawn
    v, idx = _both_windings(_tri((-1, -5, -1), (1, -5, -1), (0, -5, 1)))
    _, d = mr.render(v, idx, uni, w, h, st)
    assert np.all(d == 1.0)
    # a huge triangle around the view (vertices far outside the frustum): guard-band
    # clipping leaves the part in front, which covers the screen
    v, idx = _both_windings(_tri((-1e4, 2.0, -1e4), (1e4, 2.0, -1e4), (0.0, 2.0, 1e4)))
    _, d = mr.render(v, idx, uni, w, h, st)
    assert np.all(d[..., 0] < 1.0)
    # reaching past the far plane (100): the far part is clipped, the near part drawn
    v, idx = _both_windings(_tri((-0.5, 1.0, -0.5), (0.5, 1.0, -0.5), (0.0, 500.0, 0.3)))
    _, d = mr.render(v, idx, uni, w, h, st)
    assert 0 < (d[..., 0] < 1.0).sum() < w * h
    # degenerate (collinear) and offscreen triangles: nothing drawn
    for t in (_tri((0, 1, 0), (0.5, 1, 0), (1, 1, 0)), _tri((50, 1, 0), (51, 1, 0), (50, 1, 1))):
        v, idx = _both_windings(t)
        _, d = mr.render(v, idx, uni, w, h, st)
        assert np.all(d == 1.0)


def test_restated_stages_equal_the_reference_on_the_benchmark_scene():
    """The mesh-pass benchmark's ~80k-triangle scene at 48 x 36: the restated
    vert / frag / envmap stages and the reference's own (translated) give
    the same colour within 1e-6 and the same depth."""
    import importlib.util

    import build_ref
    import refrun
    if not build_ref.reference_available():
        pytest.skip("reference checkout not present")
    spec = importlib.util.spec_from_file_location("bench", Path(__file__).resolve().parent.parent / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    from nprush_b200 import camera
    sc, env, uni = bench.mr_scene()
    w, h = 48, 36
    vp, inv = camera.view_proj((4.0, -3.5, 2.6), (0.0, 0.0, 0.3), 0.9, w / h, up=(0.0, 0.0, 1.0))
    uni[0:16], uni[36:52] = vp, inv
    c1, d1 = mr.render(sc.vertices, sc.indices, uni, w, h, mr.RestatedStages(env, env))
    c2, d2 = mr.render(sc.vertices, sc.indices, uni, w, h, refrun.MeshStages(uni, env, env))
    np.testing.assert_allclose(c1, c2, atol=1e-6, rtol=0)
    np.testing.assert_array_equal(d1, d2)
    assert (d1[..., 0] < 1).mean() > 0.2  # the mesh covers a good part of the view
