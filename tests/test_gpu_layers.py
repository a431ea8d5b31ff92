"""The layered fit (splats, then edge / base-colour / fine-colour Bezier
layers, as the reference's viewer loop runs them) on a small synthetic target:
every layer trains, the colour layer's background is the base layer drawn
over the splats, and the finished composite approaches the target."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from scenes import camera  # noqa: E402


def synthetic_target(w, h):
    yy, xx = np.mgrid[0:h, 0:w] / max(w, h)
    rgba = np.zeros((h, w, 4), np.float32)
    rgba[..., 0] = 0.2 + 0.6 * xx
    rgba[..., 1] = 0.3 + 0.4 * yy
    rgba[..., 2] = 0.5
    rgba[..., 3] = 1.0
    disk = (xx - 0.5) ** 2 + (yy - 0.45) ** 2 < 0.22 ** 2
    rgba[disk, :3] = (0.9, 0.2, 0.1)
    depth = np.where(disk, 0.4, 1.0).astype(np.float32)
    normal = np.zeros((h, w, 4), np.float32)
    normal[disk, 2] = 1.0
    return rgba, depth, normal


def test_layered_fit_trains_every_layer():
    from nprush_b200 import build
    build.build()
    from nprush_b200.layers import LayeredFit
    w = h = 96
    rgba, depth, normal = synthetic_target(w, h)
    vp, vpi = camera(w, h, dist=1.6, fov=math.pi / 3)
    t = torch.from_numpy(rgba).cuda()
    fit = LayeredFit(t, torch.from_numpy(depth).cuda(), torch.from_numpy(normal).cuda(), vp, vpi, num_splats=512,
                     num_beziers=128, seed=3)
    assert float(fit.edge[..., 0].max()) == 1.0 and float(fit.edge[..., 0].min()) == 0.0  # the silhouette
    mse0 = float(torch.mean((fit.composite()[..., :3] - t[..., :3]) ** 2))
    before = {k: m.read_state()["beziers"].copy() for k, m in fit.bz.items()}
    for _ in range(40):
        fit.frame()
    torch.cuda.synchronize()
    # every layer's curves moved
    for k, m in fit.bz.items():
        assert not np.array_equal(m.read_state()["beziers"], before[k]), k
    # the colour layer's background is the base layer over the splats
    ref = torch.zeros_like(t)
    fit.bz["base"].render(fit.vp, w, h, ref, background=fit.splat_rgba)
    assert fit.last_background is fit.bg_after_base
    torch.testing.assert_close(ref, fit.bg_after_base)
    out = fit.composite()
    assert torch.isfinite(out).all()
    mse = float(torch.mean((out[..., :3] - t[..., :3]) ** 2))
    assert mse < 0.8 * mse0, (mse0, mse)
    fit.close()


def test_layered_fit_on_mesh_targets():
    """The reference's whole per-frame chain on a mesh: mesh pass (normals
    shading, reciprocal depth) and path-traced colour as targets, then the
    preprocessing, the splats and the three Bezier layers."""
    from nprush_b200 import build
    build.build()
    from nprush_b200 import meshes
    from nprush_b200.layers import LayeredFit, mesh_targets
    w = h = 96
    scene = meshes.concat([meshes.uv_sphere((0.0, 0.0, 0.0), 0.35, (0.8, 0.3, 0.2, 1.0), 12, 24),
                           meshes.box((0.3, 0.25, -0.2), 0.15, (0.2, 0.6, 0.8, 1.0))])
    env = meshes.sky_env(64, 32)
    t, d, n, vp, vpi = mesh_targets(scene, (1.2, -1.0, 0.6), (0.0, 0.0, 0.0), w, h, math.pi / 3, env=env,
                                    path_trace_frames=16)
    fg = d < 1.0
    assert 0.1 < float(fg.float().mean()) < 0.9                    # the mesh and the sky
    assert float((t[..., :3] - n[..., :3]).abs().max()) > 0.1       # path-traced colour, not the raster's
    assert torch.all((t * 255 - torch.round(t * 255)).abs() < 1e-3)  # 8-bit levels
    fit = LayeredFit(t, d, n, vp, vpi, num_splats=512, num_beziers=128, seed=5)
    assert float(fit.edge[..., 0].max()) == 1.0  # the silhouette from the rendered depth
    mse0 = float(torch.mean((fit.composite()[..., :3] - t[..., :3]) ** 2))
    for _ in range(40):
        fit.frame()
    torch.cuda.synchronize()
    out = fit.composite()
    assert torch.isfinite(out).all()
    mse = float(torch.mean((out[..., :3] - t[..., :3]) ** 2))
    assert mse < 0.8 * mse0, (mse0, mse)
    fit.close()
