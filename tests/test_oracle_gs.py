"""CPU checks of the Gaussian-model oracle: the fp32 analytic backward (the
port that is also the timed CPU baseline) against FP64 central differences of
the loss with the base point's discrete decisions frozen (h = 1e-4 relative)."""
import numpy as np
import pytest

import oracle as orc
from gs_scenes import gs_scene, gs_targets, gs_views


@pytest.mark.parametrize("deg,nviews,loss", [(0, 1, "l1_dssim"), (3, 2, "l1_dssim"), (0, 1, "l1"), (3, 2, "l2")])
def test_analytic_backward_matches_fp64_central_differences(deg, nviews, loss):
    n, w, h = 200, 48, 40
    p = gs_scene(n, 3 + deg, deg=deg, log_scale_mean=-3.0, spread=0.8)
    eyes = [(0.0, 0.0, 4.0), (2.5, 1.0, 3.0)][:nviews]
    vp, vpi, views = gs_views(w, h, eyes)
    tg = gs_targets(nviews, w, h, 7)
    tids = np.arange(nviews, dtype=np.uint32)
    img, nc = orc.gs_forward(p, deg, views, w, h)
    l3, dimg = orc.gs_loss(img, tg, tids, loss=loss)
    g = orc.gs_backward(p, deg, views, w, h, img, nc, dimg)
    # loss value agrees with the FP64 evaluation
    assert abs(orc.gs_loss_f64(p, deg, views, w, h, tg, tids, loss=loss) - l3[0]) < 1e-5
    rng = np.random.default_rng(0)
    touched = np.nonzero(np.abs(g[:, 0]) > 0)[0]
    assert len(touched) > 20
    gi = rng.choice(touched, 24, replace=False)
    fields = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14] + ([15, 20, 40, 59] if deg == 3 else [])
    pidx = np.array([i * 64 + f for i in gi for f in fields], np.uint32)
    cd = orc.gs_loss_cd(p, deg, views, w, h, tg, tids, pidx, loss=loss)
    an = g.reshape(-1)[pidx].astype(np.float64)
    scale = np.abs(cd).max()
    err = np.abs(an - cd)
    # relative to each value, with a floor at 1e-3 of the largest gradient
    rel = err / np.maximum(np.abs(cd), 1e-3 * scale)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert np.quantile(rel, 0.98) < 1e-3, np.quantile(rel, 0.98)


def test_adc_oracle_invariants():
    """Plain ADC restatement: prune, clone and split counts, order and state."""
    import math

    from adc_scenes import adc_case

    n = 4000
    p, m, v, grad, denom = adc_case(n, 3)
    op = 1 / (1 + np.exp(-p[:, 10].astype(np.float64)))
    keep = ~(op < 0.005)
    avg = np.where(denom > 0, grad / np.maximum(denom, 1), 0)
    cand = keep & (avg >= 2e-4)
    split = cand & (np.exp(p[:, 3:6].max(1)) > 0.01)
    for cap, seed in ((2 * n, 1), (int(keep.sum()) + 100, 2)):
        q, qm, qv, c = orc.gs_adc(p, m, v, grad, denom, cap, seed)
        budget = cap - int(keep.sum())
        dens = min(int(cand.sum()), budget)
        assert tuple(c) == (n, int(keep.sum()) + dens, dens, int((~keep).sum()))
        assert len(q) == c[1] <= cap
        # walk the parents in order and check each one's outputs
        o, rank = 0, 0
        for i in np.flatnonzero(keep):
            d = cand[i] and rank < budget
            rank += int(cand[i])
            if not d:
                assert np.array_equal(q[o], p[i]) and np.array_equal(qm[o], m[i]) and np.array_equal(qv[o], v[i])
                o += 1
            elif not split[i]:
                assert np.array_equal(q[o], p[i]) and np.array_equal(q[o + 1], p[i])
                assert np.array_equal(qm[o], m[i]) and not qm[o + 1].any() and not qv[o + 1].any()
                o += 2
            else:
                for ch in (0, 1):
                    np.testing.assert_allclose(q[o + ch, 3:6], p[i, 3:6] - math.log(1.6), atol=1e-6)
                    assert np.array_equal(q[o + ch, 6:], p[i, 6:])
                    # children within 6 sigma of the parent along every axis
                    assert np.linalg.norm(q[o + ch, :3] - p[i, :3]) <= 6 * math.sqrt(3) * np.exp(p[i, 3:6]).max()
                    assert not qm[o + ch].any() and not qv[o + ch].any()
                assert not np.array_equal(q[o, :3], q[o + 1, :3])
                o += 2
        assert o == c[1]


def _sphere_quadrature():
    """Gauss-Legendre in z (8 nodes) x 16 uniform angles: exact for the
    products of two SH of degree <= 3 (degree 6 in z, trigonometric degree
    6 in phi)."""
    z, wz = np.polynomial.legendre.leggauss(8)
    phi = 2 * np.pi * np.arange(16) / 16
    s = np.sqrt(1 - z * z)
    dirs = np.stack([np.outer(s, np.cos(phi)), np.outer(s, np.sin(phi)), np.repeat(z[:, None], 16, 1)], -1)
    w = np.repeat(wz[:, None] * (2 * np.pi / 16), 16, 1)
    return dirs.reshape(-1, 3), w.reshape(-1)


def test_sh_basis_is_orthonormal_on_the_sphere():
    """The oracle's SH table comes from the closed-form normalisations; over
    the sphere the 16 functions are orthonormal, and degree 1 carries the
    Condon-Shortley signs (-y, z, -x)."""
    dirs, w = _sphere_quadrature()
    b = orc.gs_sh(dirs)[0]
    gram = (b * w[:, None]).T @ b
    np.testing.assert_allclose(gram, np.eye(16), atol=1e-12)
    k1 = np.sqrt(3 / (4 * np.pi))
    np.testing.assert_allclose(b[:, 1:4], k1 * np.stack([-dirs[:, 1], dirs[:, 2], -dirs[:, 0]], 1), atol=1e-15)
    np.testing.assert_allclose(b[:, 0], 0.5 / np.sqrt(np.pi), atol=1e-16)


def test_sh_partials_match_central_differences():
    rng = np.random.default_rng(3)
    pts = rng.normal(size=(50, 3))
    _, gx, gy, gz = orc.gs_sh(pts)
    h = 1e-6
    for axis, g in enumerate((gx, gy, gz)):
        e = np.zeros(3)
        e[axis] = h
        fd = (orc.gs_sh(pts + e)[0] - orc.gs_sh(pts - e)[0]) / (2 * h)
        np.testing.assert_allclose(g, fd, atol=1e-7, rtol=1e-7)


def test_quaternion_rotation_and_its_gradient():
    rng = np.random.default_rng(4)
    # a quarter turn about z takes x to y
    q = np.array([np.cos(np.pi / 4), 0, 0, np.sin(np.pi / 4)])
    R, _ = orc.gs_rot(q, np.zeros(9))
    np.testing.assert_allclose(R @ [1, 0, 0], [0, 1, 0], atol=1e-15)
    for _ in range(20):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        G = rng.normal(size=(3, 3))
        R, dq = orc.gs_rot(q, G)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
        assert abs(np.linalg.det(R) - 1) < 1e-14
        # R(q) is a polynomial in q; differentiate sum G * R without renormalising
        fd = np.zeros(4)
        for k in range(4):
            e = np.zeros(4)
            e[k] = 1e-6
            fd[k] = ((G * orc.gs_rot(q + e, G)[0]).sum() - (G * orc.gs_rot(q - e, G)[0]).sum()) / 2e-6
        np.testing.assert_allclose(dq, fd, atol=1e-8)
