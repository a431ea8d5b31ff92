"""CPU checks of the Gaussian-model oracle: the fp32 analytic backward (the
port that is also the timed CPU baseline) against FP64 central differences of
the loss with the base point's discrete decisions frozen (h = 1e-4 relative)."""
import numpy as np
import pytest

import oracle as orc
from gs_scenes import gs_scene, gs_targets, gs_views


@pytest.mark.parametrize("deg,nviews", [(0, 1), (3, 2)])
def test_analytic_backward_matches_fp64_central_differences(deg, nviews):
    n, w, h = 200, 48, 40
    p = gs_scene(n, 3 + deg, deg=deg, log_scale_mean=-3.0, spread=0.8)
    eyes = [(0.0, 0.0, 4.0), (2.5, 1.0, 3.0)][:nviews]
    vp, vpi, views = gs_views(w, h, eyes)
    tg = gs_targets(nviews, w, h, 7)
    tids = np.arange(nviews, dtype=np.uint32)
    img, nc = orc.gs_forward(p, deg, views, w, h)
    l3, dimg = orc.gs_loss(img, tg, tids)
    g = orc.gs_backward(p, deg, views, w, h, img, nc, dimg)
    # loss value agrees with the FP64 evaluation
    assert abs(orc.gs_loss_f64(p, deg, views, w, h, tg, tids) - l3[0]) < 1e-5
    rng = np.random.default_rng(0)
    touched = np.nonzero(np.abs(g[:, 0]) > 0)[0]
    assert len(touched) > 20
    gi = rng.choice(touched, 24, replace=False)
    fields = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14] + ([15, 20, 40, 59] if deg == 3 else [])
    pidx = np.array([i * 64 + f for i in gi for f in fields], np.uint32)
    cd = orc.gs_loss_cd(p, deg, views, w, h, tg, tids, pidx)
    an = g.reshape(-1)[pidx].astype(np.float64)
    scale = np.abs(cd).max()
    err = np.abs(an - cd)
    # relative to each value, with a floor at 1e-3 of the largest gradient
    rel = err / np.maximum(np.abs(cd), 1e-3 * scale)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert np.quantile(rel, 0.98) < 1e-3, np.quantile(rel, 0.98)
