"""The display forwards' restatements against the reference's own render
stages (tests/golden/forward.npz: splat_forward.wgsl and bezier_forward.wgsl
vertex and fragment functions run on the host between the fixed-function
steps of oracle/forward_raster.py).

Tolerances: splat pass 2e-6 absolute (the restatement composites front to
back, the pipeline blends in draw order: two roundings of the same sums);
Bezier pass 1e-5 (the fragment's p_screen is interpolated across the quad in
the pipeline and computed at the pixel centre in the restatement)."""
from pathlib import Path

import numpy as np
import pytest

import oracle as orc

GOLD = Path(__file__).resolve().parent / "golden" / "forward.npz"
W, H = 48, 40


@pytest.fixture(scope="module")
def g():
    return np.load(GOLD)


def test_splat_pass_cleared_and_loading(g):
    s, vp = g["splat_params"], g["splat_vp"]
    c, d = orc.splat_render(s, vp, W, H)
    np.testing.assert_allclose(c, g["splat_clear_rgba"], atol=2e-6, rtol=0)
    np.testing.assert_allclose(d, g["splat_clear_depth"], atol=2e-6, rtol=0)
    lc, ld = orc.splat_render_blend(s, vp, W, H, g["splat_bg_rgba"], g["splat_bg_depth"])
    np.testing.assert_allclose(lc, g["splat_load_rgba"], atol=2e-6, rtol=0)
    np.testing.assert_allclose(ld, g["splat_load_depth"], atol=2e-6, rtol=0)


def test_fixture_covers_the_far_plane(g):
    """Splat 0 lies past the far plane and is not drawn by the pipeline;
    splat 1, just inside it, is: hiding them changes the image only for 1."""
    s, vp = g["splat_params"], g["splat_vp"]
    base, _ = orc.splat_render(s, vp, W, H)
    for k, visible in ((0, False), (1, True)):
        t = s.copy()
        t[k, 7] = 0.0
        c, _ = orc.splat_render(t, vp, W, H)
        assert (np.abs(c - base).max() > 1e-3) == visible


def test_bezier_pass_cleared_and_loading(g):
    b, vp, brush = g["bezier_params"], g["bezier_vp"], g["brush"]
    np.testing.assert_allclose(orc.bezier_render(b, vp, W, H, bg=None, brush=brush), g["bezier_clear"],
                               atol=1e-5, rtol=0)
    np.testing.assert_allclose(orc.bezier_render(b, vp, W, H, bg=g["bezier_bg"], brush=brush), g["bezier_load"],
                               atol=1e-5, rtol=0)
    assert g["bezier_clear"][..., 3].max() > 0.3  # strokes visible


def test_quad_coverage_is_watertight():
    """The two triangles of a quad (either topology) cover every pixel centre
    inside it exactly once, in both windings."""
    import forward_raster as fr
    rng = np.random.default_rng(1)
    for _ in range(20):
        x0, x1 = sorted(rng.uniform(-1.2, 1.2, 2))
        y0, y1 = sorted(rng.uniform(-1.2, 1.2, 2))
        corners = [np.array([x, y, 0.5, 1.0], np.float32) for x, y in ((x0, y1), (x0, y0), (x1, y1), (x1, y0))]
        for topo, order in (("triangle-strip", [0, 1, 2, 3]), ("triangle-list", [0, 1, 2, 2, 1, 3])):
            hits = np.zeros((H, W), np.int32)
            for tri in fr.triangles(topo, len(order)):
                r = fr.raster_triangle([corners[order[k]] for k in tri], W, H)
                if r is not None:
                    np.add.at(hits, (r[1], r[0]), 1)
            assert hits.max() <= 1


def test_reference_stages_reproduce_the_fixture(tmp_path, monkeypatch):
    """Regenerating tests/golden/forward.npz from the reference checkout gives
    the committed arrays (skipped without the checkout)."""
    import importlib.util

    import build_ref
    if not build_ref.reference_available():
        pytest.skip("reference checkout not present")
    spec = importlib.util.spec_from_file_location("mk", GOLD.parent / "make_forward_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    monkeypatch.setattr(mk, "HERE", tmp_path)
    mk.main()
    a, b = np.load(GOLD), np.load(tmp_path / "forward.npz")
    assert set(a.files) == set(b.files)
    for k in a.files:
        np.testing.assert_array_equal(a[k], b[k])
