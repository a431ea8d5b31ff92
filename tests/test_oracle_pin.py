"""Pins the oracle restatement (oracle/nps_oracle.cpp) to the reference's OWN
compute shaders, translated and compiled on the host (oracle/_ref).

The reference ships no tests, fixtures or golden vectors for this path, so the
pin is the reference code itself: both sides get the same seeded inputs and
must agree bit for bit (same fp32 operation order, no FMA contraction).
Needs the reference checkout (to build oracle/_ref); CPU only.
"""
import numpy as np
import pytest

import oracle as orc
import refrun
from conftest import requires_reference
from scenes import bezier_scene, bezier_textures, camera, splat_scene, targets

pytestmark = requires_reference


@pytest.mark.parametrize("n,w,h,seed,shape", [(64, 32, 32, 0, False), (200, 48, 40, 1, True), (1100, 64, 48, 2, False)])
def test_splat_backward_matches_reference(n, w, h, seed, shape):
    s = splat_scene(n, seed, alive=n - 7, random_shape=shape)
    vp, vpi = camera(w, h)
    tgt, depth = targets(w, h, seed + 100)
    ref = refrun.splat_backward(s, vp, vpi, tgt, depth)
    mine = orc.splat_backward(s, vp, vpi, tgt, depth)
    assert np.count_nonzero(ref) > n  # the case exercises the backward
    np.testing.assert_array_equal(mine["grads_q"], ref)
    if n > 1024:
        assert mine["tile_count"].max() == 1024  # the cap is exercised


def test_splat_backward_dense_tile_cap():
    # many tiny splats in one tile: the 1024 cap drops the highest indices
    n = 1500
    s = splat_scene(n, 5, spread=0.02, scale=(0.002, 0.004))
    vp, vpi = camera(32, 32, dist=1.2, eye=(0, 0, 1.2))
    tgt, depth = targets(32, 32, 6)
    ref = refrun.splat_backward(s, vp, vpi, tgt, depth)
    mine = orc.splat_backward(s, vp, vpi, tgt, depth)
    assert mine["tile_count"].max() == 1024
    np.testing.assert_array_equal(mine["grads_q"], ref)


def test_splat_step_matches_reference():
    n = 300
    rng = np.random.default_rng(3)
    s = splat_scene(n, 3, alive=280)
    s[5, 7] = 0.051  # near the kill threshold
    s[6, 3] = 0.0012; s[6, 12] = 0.0012; s[6, 15] = 0.001  # volume kill
    g = rng.integers(-200000, 200000, (n, 16), dtype=np.int32)
    m = rng.normal(0, 1e-3, (n, 16)).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-5, (n, 16))).astype(np.float32)
    ga = rng.random(n).astype(np.float32) * 1e-3
    for t0 in (0.0, 7.0):
        rs, rg, rm, rv, ra, rt = refrun.splat_step(s, g, m, v, t0, ga)
        ms, mg, mm, mv, ma = s.copy(), g.copy(), m.copy(), v.copy(), ga.copy()
        mt = orc.splat_step(ms, mg, mm, mv, t0, ma)
        assert mt == rt
        for a, b in ((ms, rs), (mg, rg), (mm, rm), (mv, rv), (ma, ra)):
            np.testing.assert_array_equal(a, b)


def test_splat_adc_matches_reference():
    n = 256
    rng = np.random.default_rng(4)
    s = splat_scene(n, 4, alive=None)
    dead = rng.random(n) < 0.35
    s[dead, 7] = 0.0
    s[::7, 3] = 0.002; s[::7, 12] = 0.002; s[::7, 15] = 0.002  # clone branch
    ga = (rng.random(n) * 4e-3).astype(np.float32)  # ~half above 25 * 5e-5
    ga[dead] = (rng.random(dead.sum()) * 4e-3).astype(np.float32)  # stale values on dead slots
    m = rng.normal(0, 1e-3, (n, 16)).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-5, (n, 16))).astype(np.float32)
    rs, rm, rv, ra = refrun.splat_adc(s, m, v, 50.0, ga)
    ms, mm, mv, ma = s.copy(), m.copy(), v.copy(), ga.copy()
    orc.splat_adc(ms, mm, mv, 50.0, ma)
    assert (rs[:, 7] >= 0.05).sum() > (s[:, 7] >= 0.05).sum()  # slots were filled
    for a, b in ((ms, rs), (mm, rm), (mv, rv), (ma, ra)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("mode,max_width,bgp", [(1.0, 0.0, 0.0), (1.0, 0.012, 0.3), (0.0, 0.0, 0.0)])
def test_bezier_backward_matches_reference(mode, max_width, bgp):
    n, w, h = 96, 48, 32
    b = bezier_scene(n, 7, alive=90)
    vp, vpi = camera(w, h, dist=1.4)
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, 8)
    uni = refrun.bezier_uniforms(vp, vpi, mode=mode, max_width=max_width, bg_penalty=bgp)
    adc0 = np.zeros(2 * n, np.float32)
    adc0[n:] = 0.25
    rg, radc, rpl = refrun.bezier_backward(b, uni, tgt, depth, bg, bgd, nrm, adc=adc0)
    la = adc0[n:].copy()
    mine = orc.bezier_backward(b, vp, uni[16:22], tgt, depth, bg, bgd, nrm, loss_accum=la)
    assert np.count_nonzero(rg) > n
    np.testing.assert_array_equal(mine["grads_q"], rg)
    np.testing.assert_array_equal(mine["pixel_loss"], rpl)
    np.testing.assert_array_equal(mine["loss_accum"], radc[n:])


def test_bezier_step_matches_reference():
    n = 200
    rng = np.random.default_rng(9)
    b = bezier_scene(n, 9, alive=190)
    b[3, 19] = 0.0011  # prune by alpha
    b[4, 3] = 0.0009   # prune by width
    b[5, 0:16:4] = 30.0  # far right: offscreen kill
    vp, vpi = camera(64, 64)
    g = rng.integers(-200000, 200000, (n, 18), dtype=np.int32)
    m = rng.normal(0, 1e-3, (n, 18)).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-5, (n, 18))).astype(np.float32)
    ga = rng.random(n).astype(np.float32) * 1e-3
    for max_width, no_kill in ((0.0, 0.0), (0.012, 1.0)):
        uni = refrun.bezier_uniforms(vp, vpi, max_width=max_width, prune_alpha=0.0, prune_width=0.0)
        rb, rg, rm, rv, ra, rt = refrun.bezier_step(b, g, m, v, 3.0, 4096.0, no_kill, ga, uni)
        mb, mg, mm, mv, ma = b.copy(), g.copy(), m.copy(), v.copy(), ga.copy()
        mt = orc.bezier_step(mb, mg, mm, mv, 3.0, 4096.0, no_kill, ma, vp, uni[16:22])
        assert mt == rt
        for a, c in ((mb, rb), (mg, rg), (mm, rm), (mv, rv), (ma, ra)):
            np.testing.assert_array_equal(a, c)


@pytest.mark.parametrize("no_kill", [0.0, 1.0])
def test_bezier_adc_matches_reference(no_kill):
    n = 300
    rng = np.random.default_rng(11)
    b = bezier_scene(n, 11)
    b[rng.random(n) < 0.3, 19] = 0.0
    b[7, 0:16:4] = 40.0  # offscreen
    vp, vpi = camera(256, 256, dist=1.5)
    ga = (rng.random(n) * 0.02).astype(np.float32)
    la = (rng.random(n) * 0.1).astype(np.float32)
    pl = np.zeros(512 * 512, np.int32)
    pl[rng.integers(0, 512 * 512, 3000)] = rng.integers(1, 10000, 3000)
    m = rng.normal(0, 1e-3, (n, 18)).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-5, (n, 18))).astype(np.float32)
    uni = refrun.bezier_uniforms(vp, vpi)
    rb, rm, rv, rga, rla, rpl = refrun.bezier_adc(b, m, v, 77.0, no_kill, ga, la, pl, uni)
    mb, mm, mv, mga, mla, mpl = b.copy(), m.copy(), v.copy(), ga.copy(), la.copy(), pl.copy()
    orc.bezier_adc(mb, mm, mv, 77.0, no_kill, mga, mla, mpl, vp, vpi)
    for a, c in ((mb, rb), (mm, rm), (mv, rv), (mga, rga), (mla, rla), (mpl, rpl)):
        np.testing.assert_array_equal(a, c)
