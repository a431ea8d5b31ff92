"""GPU parity of the reference-semantics Bezier path against the CPU oracle
(oracle/nps_oracle.cpp, pinned bit-exact to the reference's own
bezier_{backward,step,adc}.wgsl by test_oracle_pin.py).

Tolerances: composite 1e-5 absolute; i32 gradient sums (per-pair truncation,
as for splats) bit-exact: the curve kernels use only +, -, *, / and sqrt,
each correctly rounded and unfused (--fmad=false), as the oracle does, and
integer sums do not depend on their order; pixel_loss (per-pixel i32, one term per
pixel) within 1 unit or 1e-4 relative; loss_accum 1e-4 relative (the reference
adds it with a non-atomic read-modify-write, a race; here it is an atomic
float sum); Adam step bit-exact; ADC bit-exact except the clone jitter (sinf).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as orc  # noqa: E402
from scenes import bezier_scene, bezier_textures, camera  # noqa: E402


@pytest.fixture(scope="module")
def cls():
    from nprush_b200 import build
    build.build()
    from nprush_b200.bezier import GpuBezierOptimizerManager
    return GpuBezierOptimizerManager


def uni6(mode, max_width, pa, pw, bgp):
    return np.array([mode, max_width, pa, pw, bgp, 0.0], np.float32)


@pytest.mark.parametrize("n,w,h,mode,max_width,bgp,seed", [(96, 48, 32, 1.0, 0.0, 0.0, 7), (400, 64, 64, 1.0, 0.012, 0.3, 8),
                                                        (300, 80, 48, 0.0, 0.0, 0.0, 9), (2600, 32, 32, 1.0, 0.0, 0.0, 10)])
def test_backward_matches_oracle(cls, n, w, h, mode, max_width, bgp, seed):
    b = bezier_scene(n, seed, alive=n - 5)
    vp, vpi = camera(w, h, dist=1.4)
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, seed + 1)
    m = cls(n, init=b)
    m.write_vp(vp, vpi)
    m.write_mode(mode)
    m.write_max_width(max_width)
    m.write_bg_penalty(bgp)
    la0 = np.full(n, 0.25, np.float32)
    m.write_state(loss_accum=la0)
    m.set_backward_target(tgt, depth, bg, bgd, nrm, w, h)
    img = torch.zeros((1, h, w, 4), device="cuda")
    m.backward(out_rgbd=img)
    st = m.read_state()
    ref = orc.bezier_backward(b, vp, uni6(mode, max_width, 0, 0, bgp), tgt, depth, bg, bgd, nrm,
                              loss_accum=la0.copy())
    np.testing.assert_allclose(img.cpu().numpy()[0], ref["image"], atol=1e-5, rtol=0)
    assert ref["terms"].sum() > 0
    g, r = st["grads"].astype(np.float64), ref["grads_q"].astype(np.float64)
    assert np.abs(r).sum() > 0
    rel = np.linalg.norm(g - r) / np.linalg.norm(r)
    assert rel <= 1e-4, rel
    diff = np.abs(g - r)
    t = ref["terms"].astype(np.float64)[:, None]
    assert (diff == 0).all(), ((diff != 0).mean(), (diff / (t + 1)).max())
    pl, rpl = st["pixel_loss"].astype(np.int64), ref["pixel_loss"].astype(np.int64)
    assert (np.abs(pl - rpl) <= np.maximum(1, 1e-4 * np.abs(rpl))).all()
    np.testing.assert_allclose(st["loss_accum"], ref["loss_accum"], rtol=1e-4, atol=1e-6)
    if n >= 2600:
        assert ref["tile_count"].max() == 1024


def test_step_bit_exact(cls):
    n = 500
    rng = np.random.default_rng(9)
    b = bezier_scene(n, 9, alive=480)
    b[3, 19] = 0.0011
    b[4, 3] = 0.0009
    b[5, 0:16:4] = 30.0
    vp, vpi = camera(64, 48)
    g = rng.integers(-200000, 200000, (n, 18), dtype=np.int32)
    m0 = rng.normal(0, 1e-3, (n, 18)).astype(np.float32)
    v0 = np.abs(rng.normal(0, 1e-5, (n, 18))).astype(np.float32)
    ga = (rng.random(n) * 1e-3).astype(np.float32)
    for max_width, no_kill in ((0.0, False), (0.012, True)):
        mg = cls(n, init=b)
        mg.write_vp(vp, vpi)
        mg.write_max_width(max_width)
        mg.write_no_kill(no_kill)
        tgt, depth, bg, bgd, nrm = bezier_textures(64, 48, 3)
        mg.set_backward_target(tgt, depth, bg, bgd, nrm, 64, 48)  # pixel_count = 64 * 48
        mg.write_state(grads=g, adam_m=m0, adam_v=v0, adam_t=3.0, grad_accum=ga)
        mg.step()
        st = mg.read_state()
        rb, rg, rm, rv, ra = b.copy(), g.copy(), m0.copy(), v0.copy(), ga.copy()
        t = orc.bezier_step(rb, rg, rm, rv, 3.0, 64.0 * 48.0, 1.0 if no_kill else 0.0, ra, vp,
                            uni6(1.0, max_width, 0, 0, 0))
        assert st["adam_t"] == t
        np.testing.assert_array_equal(st["beziers"], rb)
        np.testing.assert_array_equal(st["adam_m"], rm)
        np.testing.assert_array_equal(st["adam_v"], rv)
        np.testing.assert_array_equal(st["grad_accum"], ra)
        assert (st["grads"] == 0).all()


@pytest.mark.parametrize("no_kill,n,seed", [(False, 300, 11), (True, 300, 12), (False, 3000, 13)])
def test_adc_matches_oracle(cls, no_kill, n, seed):
    rng = np.random.default_rng(seed)
    b = bezier_scene(n, seed)
    b[rng.random(n) < 0.3, 19] = 0.0
    b[7, 0:16:4] = 40.0
    vp, vpi = camera(256, 256, dist=1.5)
    ga = (rng.random(n) * 0.02).astype(np.float32)
    la = (rng.random(n) * 0.1).astype(np.float32)
    pl = np.zeros(512 * 512, np.int32)
    pl[rng.integers(0, 512 * 512, 3000)] = rng.integers(1, 10000, 3000)
    m0 = rng.normal(0, 1e-3, (n, 18)).astype(np.float32)
    v0 = np.abs(rng.normal(0, 1e-5, (n, 18))).astype(np.float32)
    mg = cls(n, init=b)
    mg.write_vp(vp, vpi)
    mg.write_no_kill(no_kill)
    mg.write_state(adam_m=m0, adam_v=v0, adam_t=77.0, grad_accum=ga, loss_accum=la, pixel_loss=pl)
    mg.adc()
    st = mg.read_state()
    rb, rm, rv, rga, rla, rpl = b.copy(), m0.copy(), v0.copy(), ga.copy(), la.copy(), pl.copy()
    orc.bezier_adc(rb, rm, rv, 77.0, 1.0 if no_kill else 0.0, rga, rla, rpl, vp, vpi)
    np.testing.assert_array_equal(st["adam_m"], rm)
    np.testing.assert_array_equal(st["adam_v"], rv)
    np.testing.assert_array_equal(st["grad_accum"], rga)
    np.testing.assert_array_equal(st["loss_accum"], rla)
    np.testing.assert_array_equal(st["pixel_loss"], rpl)
    # alpha, width, softness and colour are exact, so every kill, clone, split
    # and spawn went to the same slot; control points agree up to the clone
    # jitter (fract(sin(seed * k) * 43758.5453) - 0.5) * 0.001, where CUDA's
    # sinf (2 ulp) and glibc's differ by enough, at these seeds, to wrap fract
    # in about 1% of evaluations: such elements differ by at most 0.001.
    np.testing.assert_array_equal(st["beziers"][:, 16:20], rb[:, 16:20])
    np.testing.assert_array_equal(st["beziers"][:, [3, 7]], rb[:, [3, 7]])
    diff = np.abs(st["beziers"][:, :16] - rb[:, :16])
    off = diff > 2e-5
    assert off.mean() <= 0.02, off.mean()
    assert (diff[off] <= 0.0011).all(), diff.max()
    assert mg.stats()["adc_clones"] + mg.stats()["spawns"] > 0


def test_dispatch_runs_and_learns(cls):
    """Five reference dispatches of a colour-mode layer: the composite error drops."""
    n, w, h = 2000, 96, 96
    from nprush_b200.bezier import reference_init
    b = reference_init(n, 3)
    vp, vpi = camera(w, h, dist=1.5, eye=(0.0, 0.0, 1.5))
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, 4)
    tgt[..., :3] = 0.8  # a flat target the strokes can match
    m = cls(n, init=b)
    m.write_vp(vp, vpi)
    m.write_mode(1.0)
    m.set_backward_target(tgt, depth, bg, bgd, nrm, w, h)
    img = torch.zeros((1, h, w, 4), device="cuda")
    m.backward(out_rgbd=img)
    e0 = float(np.abs(img.cpu().numpy()[0, ..., :3] - 0.8).mean())
    for _ in range(60):
        m.dispatch()
    m.backward(out_rgbd=img)
    e1 = float(np.abs(img.cpu().numpy()[0, ..., :3] - 0.8).mean())
    assert e1 < e0, (e0, e1)


def test_separate_vp_writes_equal_the_combined_write(cls):
    """writeVPMatrix then writeVPInvMatrix (either order) leaves the same
    uniforms as writing both at once: the dispatched states are bit-identical."""
    n, w, h = 500, 64, 48
    from nprush_b200.bezier import reference_init
    b = reference_init(n, 5)
    vp, vpi = camera(w, h, dist=1.5, eye=(0.3, -0.2, 1.5))
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, 6)
    states = []
    for order in ("both", "vp_first", "inv_first"):
        m = cls(n, init=b)
        if order == "both":
            m.write_vp(vp, vpi)
        elif order == "vp_first":
            m.writeVPMatrix(vp)
            m.writeVPInvMatrix(vpi)
        else:
            m.write_vp_inv_matrix(vpi)
            m.write_vp_matrix(vp)
        m.write_mode(1.0)
        m.set_backward_target(tgt, depth, bg, bgd, nrm, w, h)
        for _ in range(3):
            m.dispatch()
        states.append(m.read_state())
        m.close()
    for st in states[1:]:
        for k in ("beziers", "adam_m", "adam_v", "grad_accum"):
            np.testing.assert_array_equal(st[k], states[0][k])
