"""The oracle's per-primitive term counts (the bound of the GPU parity tests
for the reference's i32 gradient sums): a splat or curve with no backward term
(no pixel where its alpha >= 0.001) has an all-zero gradient row, one with
terms has a count no larger than the pixels of its capped tile lists, and the
counts of several views add up.  CPU only."""
import numpy as np

import oracle as orc
from scenes import bezier_scene, bezier_textures, camera, splat_scene, targets


def test_splat_terms_bound_the_gradient_rows():
    n, w, h = 800, 48, 40
    s = splat_scene(n, 41, alive=n - 20)
    vp, vpi = camera(w, h)
    tgt, depth = targets(w, h, 42)
    r = orc.splat_backward(s, vp, vpi, tgt, depth)
    terms, g = r["terms"], r["grads_q"]
    assert terms.sum() > 0 and (terms > 0).sum() < n  # some splats contribute, some do not
    assert (g[terms == 0] == 0).all()
    assert (terms[n - 20:] == 0).all()  # dead splats (opacity 0) are never binned
    assert terms.max() <= w * h


def test_splat_terms_add_over_views():
    n, w, h = 300, 32, 32
    s = splat_scene(n, 43)
    cams = [camera(w, h, eye=e) for e in ((0.3, 0.4, 1.6), (-1.2, 0.2, 1.0))]
    tg = [targets(w, h, 44 + k) for k in range(2)]
    acc = np.zeros(n, np.uint32)
    single = []
    for (vp, vpi), (t, d) in zip(cams, tg):
        orc.splat_backward(s, vp, vpi, t, d, terms=acc)
        single.append(orc.splat_backward(s, vp, vpi, t, d)["terms"])
    np.testing.assert_array_equal(acc, single[0] + single[1])


def test_bezier_terms_bound_the_gradient_rows():
    n, w, h = 200, 48, 32
    b = bezier_scene(n, 45, alive=n - 5)
    vp, _ = camera(w, h, dist=1.4)
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, 46)
    uni = np.array([1.0, 0.0, 0.0, 0.0, 0.0, 0.0], np.float32)
    r = orc.bezier_backward(b, vp, uni, tgt, depth, bg, bgd, nrm)
    terms, g = r["terms"], r["grads_q"]
    assert terms.sum() > 0
    assert (g[terms == 0] == 0).all()
    assert terms.max() <= w * h
