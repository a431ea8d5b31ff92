"""GPU parity of the headless display forwards (splat_forward.wgsl,
bezier_forward.wgsl) against the oracle's restatements: fp32 composites to
1e-5 absolute per channel (the reference's rgba8 targets are not emulated)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as orc  # noqa: E402
from scenes import bezier_scene, bezier_textures, camera, splat_scene  # noqa: E402


@pytest.mark.parametrize("n,w,h,seed", [(300, 64, 48, 1), (3000, 128, 96, 2)])
def test_splat_render_matches_oracle(n, w, h, seed):
    from nprush_b200.splat import GpuSplatOptimizerManager
    s = splat_scene(n, seed, alive=n - 11, random_shape=True)
    vp, _ = camera(w, h)
    m = GpuSplatOptimizerManager(n, init=s)
    rgba = torch.zeros((h, w, 4), device="cuda")
    dep = torch.zeros((h, w, 4), device="cuda")
    m.render(vp, w, h, rgba, dep)
    r_rgba, r_dep = orc.splat_render(s, vp, w, h)
    np.testing.assert_allclose(rgba.cpu().numpy(), r_rgba, atol=1e-5, rtol=0)
    np.testing.assert_allclose(dep.cpu().numpy(), r_dep, atol=1e-5, rtol=0)
    assert np.abs(r_rgba[..., :3] - 0.05).max() > 0.1  # splats visible


@pytest.mark.parametrize("n,w,h,seed,use_bg,use_brush", [(200, 64, 64, 3, False, False), (800, 96, 80, 4, True, True)])
def test_bezier_render_matches_oracle(n, w, h, seed, use_bg, use_brush):
    from nprush_b200.bezier import GpuBezierOptimizerManager
    b = bezier_scene(n, seed)
    vp, _ = camera(w, h, dist=1.4)
    _, _, bg, _, _ = bezier_textures(w, h, seed + 1)
    bg[..., 3] = 1.0
    rng = np.random.default_rng(seed)
    brush = rng.random((16, 32)).astype(np.float32) if use_brush else None
    m = GpuBezierOptimizerManager(n, init=b)
    out = torch.zeros((h, w, 4), device="cuda")
    m.render(vp, w, h, out, background=torch.from_numpy(bg).cuda() if use_bg else None,
             brush=torch.from_numpy(brush).cuda() if use_brush else None)
    ref = orc.bezier_render(b, vp, w, h, bg=bg if use_bg else None, brush=brush)
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=1e-5, rtol=0)
    assert ref[..., 3].max() > 0.3  # strokes visible


def test_forward_pipeline_managers():
    """GpuSplatForwardPipelineManager / GpuBezierForwardPipelineManager
    (writeVPMatrix, setTarget, dispatch) against the oracle: the cleared and
    the loading splat pass, the cleared and the loading Bezier pass."""
    from nprush_b200._lib import NpsError
    from nprush_b200.bezier import GpuBezierForwardPipelineManager, GpuBezierOptimizerManager
    from nprush_b200.splat import GpuSplatForwardPipelineManager, GpuSplatOptimizerManager
    w, h = 80, 64
    s = splat_scene(500, 5, alive=480, random_shape=True)
    vp, _ = camera(w, h)
    fwd = GpuSplatForwardPipelineManager(GpuSplatOptimizerManager(500, init=s))
    with pytest.raises(NpsError):
        fwd.dispatch(True)
    rgba = torch.zeros((h, w, 4), device="cuda")
    dep = torch.zeros((h, w, 4), device="cuda")
    fwd.writeVPMatrix(vp)
    fwd.setTarget(rgba, dep, w, h)
    fwd.dispatch(True)
    r_rgba, r_dep = orc.splat_render(s, vp, w, h)
    np.testing.assert_allclose(rgba.cpu().numpy(), r_rgba, atol=1e-5, rtol=0)
    np.testing.assert_allclose(dep.cpu().numpy(), r_dep, atol=1e-5, rtol=0)
    # the loading pass (the reference's default): blended over the current
    # contents, checked against the fragment-by-fragment draw-order blend
    rng = np.random.default_rng(9)
    c0 = rng.random((h, w, 4)).astype(np.float32)
    d0 = rng.random((h, w, 4)).astype(np.float32)
    rgba.copy_(torch.from_numpy(c0))
    dep.copy_(torch.from_numpy(d0))
    fwd.dispatch()
    want_c, want_d = orc.splat_render_blend(s, vp, w, h, c0, d0)
    np.testing.assert_allclose(rgba.cpu().numpy(), want_c, atol=1e-5, rtol=0)
    np.testing.assert_allclose(dep.cpu().numpy(), want_d, atol=1e-5, rtol=0)

    b = bezier_scene(400, 6)
    vp, _ = camera(w, h, dist=1.4)
    brush = np.random.default_rng(6).random((16, 32)).astype(np.float32)
    bfwd = GpuBezierForwardPipelineManager(GpuBezierOptimizerManager(400, init=b), brush=torch.from_numpy(brush).cuda())
    out = torch.full((h, w, 4), 0.7, device="cuda")
    bfwd.writeVPMatrix(vp)
    bfwd.setTarget(out, w, h)
    bfwd.dispatch()  # cleared
    np.testing.assert_allclose(out.cpu().numpy(), orc.bezier_render(b, vp, w, h, bg=None, brush=brush), atol=1e-5, rtol=0)
    _, _, bg, _, _ = bezier_textures(w, h, 7)
    bg[..., 3] = 1.0
    out.copy_(torch.from_numpy(bg))
    bfwd.dispatch(clear=False)
    np.testing.assert_allclose(out.cpu().numpy(), orc.bezier_render(b, vp, w, h, bg=bg, brush=brush), atol=1e-5, rtol=0)


def test_forwards_match_the_reference_pipelines():
    """Kernels against tests/golden/forward.npz (the reference's own vertex
    and fragment stages between restated fixed-function steps): cleared and
    loading passes of both forwards, 1e-5 absolute; the splat past the far
    plane is not drawn."""
    from pathlib import Path

    from nprush_b200.bezier import GpuBezierOptimizerManager
    from nprush_b200.splat import GpuSplatOptimizerManager
    g = np.load(Path(__file__).resolve().parent / "golden" / "forward.npz")
    w, h = 48, 40
    s = g["splat_params"]
    m = GpuSplatOptimizerManager(s.shape[0], init=s)
    c = torch.zeros((h, w, 4), device="cuda")
    d = torch.zeros((h, w, 4), device="cuda")
    m.render(g["splat_vp"], w, h, c, d)
    np.testing.assert_allclose(c.cpu().numpy(), g["splat_clear_rgba"], atol=1e-5, rtol=0)
    np.testing.assert_allclose(d.cpu().numpy(), g["splat_clear_depth"], atol=1e-5, rtol=0)
    c.copy_(torch.from_numpy(g["splat_bg_rgba"]))
    d.copy_(torch.from_numpy(g["splat_bg_depth"]))
    m.render(g["splat_vp"], w, h, c, d, load=True)
    np.testing.assert_allclose(c.cpu().numpy(), g["splat_load_rgba"], atol=1e-5, rtol=0)
    np.testing.assert_allclose(d.cpu().numpy(), g["splat_load_depth"], atol=1e-5, rtol=0)
    b = g["bezier_params"]
    bm = GpuBezierOptimizerManager(b.shape[0], init=b)
    brush = torch.from_numpy(g["brush"]).cuda()
    out = torch.zeros((h, w, 4), device="cuda")
    bm.render(g["bezier_vp"], w, h, out, brush=brush)
    np.testing.assert_allclose(out.cpu().numpy(), g["bezier_clear"], atol=1e-5, rtol=0)
    bm.render(g["bezier_vp"], w, h, out, background=torch.from_numpy(g["bezier_bg"]).cuda(), brush=brush)
    np.testing.assert_allclose(out.cpu().numpy(), g["bezier_load"], atol=1e-5, rtol=0)
