"""Scene files (nprush_b200/scene.py) with the real managers: a run saved
mid-way and restored into fresh managers continues bit for bit like the run
that never stopped, through the ADC schedule (the restored stepCount)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from scenes import bezier_scene, bezier_textures, camera, splat_scene, targets  # noqa: E402


@pytest.fixture(scope="module")
def lib():
    from nprush_b200 import build
    build.build()
    from nprush_b200 import scene
    return scene


def _same(a, b, keys):
    for k in keys:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_splat_run_resumes_from_scene(lib, tmp_path):
    from nprush_b200.splat import GpuSplatOptimizerManager as M
    n, w, h = 600, 48, 48
    s = splat_scene(n, 12, alive=450)
    vp, vpi = camera(w, h)
    tgt, depth = targets(w, h, 13)
    a = M(n, init=s)
    a.write_splat_vp_matrix(vp, vpi)
    a.set_backward_target(tgt, depth, w, h)
    for _ in range(20):
        a.dispatch()
    lib.write_scene(tmp_path / "s.npsc", splat_opt=a, cameras=(vp, vpi), meta={"width": w, "height": h})
    sc = lib.read_scene(tmp_path / "s.npsc")
    b = M(n, init=False)
    sc.restore_splats(b)
    b.write_splat_vp_matrix(sc["cameras.view_proj"][0], sc["cameras.inv_view_proj"][0])
    b.set_backward_target(tgt, depth, w, h)
    _same(a.read_state(), b.read_state(), ("splats", "adam_m", "adam_v", "grad_accum", "grads"))
    for _ in range(8):  # through the ADC at dispatch 25
        a.dispatch()
        b.dispatch()
    sa, sb = a.read_state(), b.read_state()
    _same(sa, sb, ("splats", "adam_m", "adam_v", "grad_accum", "grads"))
    assert sa["adam_t"] == sb["adam_t"]
    assert a.stats()["step_count"] == b.stats()["step_count"] == 28


def test_bezier_run_resumes_from_scene(lib, tmp_path):
    from nprush_b200.bezier import GpuBezierOptimizerManager as M
    from nprush_b200.bezier import reference_init
    n, w, h = 800, 64, 64
    vp, vpi = camera(w, h, dist=1.5, eye=(0.0, 0.0, 1.5))
    tgt, depth, bg, bgd, nrm = bezier_textures(w, h, 4)

    def setup(m):
        m.write_vp(vp, vpi)
        m.write_mode(1.0)
        m.set_adc_period(10)
        m.set_backward_target(tgt, depth, bg, bgd, nrm, w, h)

    a = M(n, init=reference_init(n, 3))
    setup(a)
    for _ in range(7):
        a.dispatch()
    lib.write_scene(tmp_path / "b.npsc", bezier_opt=a)
    b = M(n, init=False)
    lib.read_scene(tmp_path / "b.npsc").restore_beziers(b)
    setup(b)
    for _ in range(5):  # through the ADC at dispatch 10
        a.dispatch()
        b.dispatch()
    sa, sb = a.read_state(), b.read_state()
    _same(sa, sb, ("beziers", "adam_m", "adam_v", "grad_accum", "grads", "pixel_loss"))
    # loss_accum is a float sum of per-tile contributions added with atomics (the reference
    # adds them without, bezier_backward.wgsl:562): its last bit depends on the order in
    # which the tiles arrive, run to run
    np.testing.assert_allclose(sa["loss_accum"], sb["loss_accum"], rtol=1e-6, atol=0)


def test_gaussian_run_resumes_from_scene(lib, tmp_path):
    from gs_scenes import gs_scene, gs_targets, gs_views
    from nprush_b200.gaussians import GaussianTrainer
    n, w, h = 1024, 64, 64
    p = gs_scene(n, 2, deg=1, log_scale_mean=-3.5)
    vp, vpi, _ = gs_views(w, h)
    tg = gs_targets(1, w, h, 3)
    tids = np.zeros(1, np.uint32)

    def setup(t):
        t.set_deterministic(True)
        t.set_targets(tg)
        t.set_views(vp, vpi, tids)

    a = GaussianTrainer(n, sh_degree=1, params=p)
    setup(a)
    for _ in range(3):
        a.train_step()
    lib.write_scene(tmp_path / "g.npsc", trainer=a)
    sc = lib.read_scene(tmp_path / "g.npsc")
    assert sc.meta["gaussians.step"] == 3 and sc.meta["gaussians.sh_degree"] == 1
    b = GaussianTrainer(n, sh_degree=1)
    sc.restore_gaussians(b)
    setup(b)
    for _ in range(2):
        a.train_step()
        b.train_step()
    _same(a.read_state(), b.read_state(), ("params", "adam_m", "adam_v"))
