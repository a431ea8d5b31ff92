"""CPU checks of the display-forward restatements (no graphics stack here, so
the render pipelines themselves cannot run): the splat pass blended fragment
by fragment in draw order, as the pipeline's blend state does, equals the
front-to-back compositing form on cleared attachments."""
import numpy as np
import pytest

import oracle as orc
from scenes import camera, splat_scene


@pytest.mark.parametrize("n,w,h,seed", [(300, 64, 48, 1), (2000, 96, 80, 2)])
def test_draw_order_blend_equals_front_to_back(n, w, h, seed):
    s = splat_scene(n, seed, alive=n - 7, random_shape=True)
    vp, _ = camera(w, h)
    rgba, dep = orc.splat_render(s, vp, w, h)
    c0 = np.tile(np.array([0.05, 0.05, 0.05, 1.0], np.float32), (h, w, 1))
    d0 = np.ones((h, w, 4), np.float32)
    c1, d1 = orc.splat_render_blend(s, vp, w, h, c0, d0)
    # two evaluation orders of the same blend equation: float rounding only
    np.testing.assert_allclose(c1, rgba, atol=2e-6, rtol=0)
    np.testing.assert_allclose(d1, dep, atol=2e-6, rtol=0)
    assert np.abs(rgba[..., :3] - 0.05).max() > 0.1  # splats visible


def test_blend_over_loaded_contents():
    """Over arbitrary starting contents the pass keeps uncovered pixels as
    they were and, where splats cover, leaves the alpha at or above its
    starting value (alpha = a + dst.a (1 - a))."""
    n, w, h = 400, 64, 64
    s = splat_scene(n, 3, random_shape=True)
    vp, _ = camera(w, h)
    rng = np.random.default_rng(4)
    c0 = rng.random((h, w, 4)).astype(np.float32)
    d0 = rng.random((h, w, 4)).astype(np.float32)
    c1, d1 = orc.splat_render_blend(s, vp, w, h, c0, d0)
    covered = np.abs(orc.splat_render_blend(s, vp, w, h, np.zeros_like(c0))[0][..., 3]) > 0
    assert covered.any() and (~covered).any()
    np.testing.assert_array_equal(c1[~covered], c0[~covered])
    np.testing.assert_array_equal(d1[~covered], d0[~covered])
    assert np.all(c1[covered][:, 3] >= c0[covered][:, 3] - 1e-7)
