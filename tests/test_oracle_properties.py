"""Property tests of the splat oracle (the reference ships none): an invisible
splat contributes nothing, splats with disjoint footprints can be renumbered
without changing anything but the order of their gradient rows, and a single
splat seen head-on gives the closed-form composite at the pixel on its axis.
The GPU kernels are checked against this oracle elsewhere.  CPU only."""
import math

import numpy as np

import oracle as orc
from scenes import camera, splat_scene, targets


def test_invisible_splat_contributes_nothing():
    n, w, h = 200, 40, 32
    s = splat_scene(n, 51)
    vp, vpi = camera(w, h)
    tgt, depth = targets(w, h, 52)
    base = orc.splat_backward(s, vp, vpi, tgt, depth)
    s2 = np.concatenate([s, s[:1]])
    s2[-1, 7] = 0.004  # opacity below the binning cut (0.005): never on a tile list
    r = orc.splat_backward(s2, vp, vpi, tgt, depth)
    np.testing.assert_array_equal(r["image"], base["image"])
    np.testing.assert_array_equal(r["grads_q"][:n], base["grads_q"])
    assert (r["grads_q"][n] == 0).all() and r["terms"][n] == 0


def _two_far_apart(seed):
    s = splat_scene(2, seed, scale=(0.02, 0.03))
    s[0, 0:3] = (-0.55, 0.35, 0.0)
    s[1, 0:3] = (0.55, -0.35, 0.0)
    return s


def test_disjoint_splats_renumber_with_their_gradients():
    w, h = 64, 48
    s = _two_far_apart(53)
    vp, vpi = camera(w, h, eye=(0.0, 0.0, 1.6))
    tgt, depth = targets(w, h, 54)
    a = orc.splat_backward(s, vp, vpi, tgt, depth)
    b = orc.splat_backward(s[::-1].copy(), vp, vpi, tgt, depth)
    assert (a["terms"] > 0).all()
    # no tile holds both splats: the lists are the same after renumbering
    np.testing.assert_array_equal(a["image"], b["image"])
    np.testing.assert_array_equal(a["grads_q"], b["grads_q"][::-1])


def test_single_splat_head_on_closed_form():
    w = h = 33  # odd: the centre pixel's centre is the image centre, NDC (0, 0)
    d = 2.0
    s = np.zeros((1, 16), np.float32)
    s[0, 3] = s[0, 12] = s[0, 15] = 0.05  # sx, sy, sz
    s[0, 4:7] = (0.9, 0.4, 0.1)           # colour
    s[0, 7] = 0.6                         # opacity
    s[0, 8] = 1.0                         # identity rotation
    s[0, 13], s[0, 14] = 2.0, 0.5         # shape a, b
    vp, vpi = camera(w, h, eye=(0.0, 0.0, d))
    tgt, depth = targets(w, h, 55)
    img = orc.splat_backward(s, vp, vpi, tgt, depth)["image"]
    c = h // 2
    # r = sqrt(max(0, 1e-4)) = 0.01 at the centre; alpha = opacity * exp(-b r^a)
    f = np.float32
    alpha = min(max(f(0.6) * f(math.exp(-0.5 * 0.01 ** 2.0)), f(0.0)), f(0.999))
    view_depth = f(1.0) - f(0.1) / f(d)  # clip w = distance to the camera
    expect_rgb = f(alpha) * s[0, 4:7] + (f(1.0) - f(alpha)) * f(0.05)
    expect_d = f(alpha) * view_depth + (f(1.0) - f(alpha))
    np.testing.assert_allclose(img[c, c, :3], expect_rgb, rtol=0, atol=2e-6)
    np.testing.assert_allclose(img[c, c, 3], expect_d, rtol=0, atol=2e-6)
    # symmetric footprint: the pixels left and right of the centre see the same alpha
    np.testing.assert_allclose(img[c, c - 3], img[c, c + 3], rtol=0, atol=2e-6)
    np.testing.assert_allclose(img[c - 3, c], img[c + 3, c], rtol=0, atol=2e-6)
