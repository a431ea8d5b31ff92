"""GPU parity of the Gaussian trainer against the CPU oracle
(oracle/nps_oracle_gs.cpp), whose analytic backward is itself checked against
FP64 central differences (test_oracle_gs.py).

Tolerances: rendered images 1e-5 absolute per channel; loss 1e-5 relative;
dL/dimage 1e-6 absolute (its entries are ~1/(3HW)); parameter gradients 1e-4
relative (relative L2 over all gradients, and per value against
max(|ref|, 1e-3 * max|ref|) at the 99th percentile, since float atomics sum
the per-pixel terms in another order); Adam 1e-6 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as orc  # noqa: E402
from gs_scenes import gs_scene, gs_targets, gs_views  # noqa: E402


@pytest.fixture(scope="module")
def trainer_cls():
    from nprush_b200 import build
    build.build()
    from nprush_b200.gaussians import GaussianTrainer
    return GaussianTrainer


def run_gpu(cls, p, deg, vp, vpi, tg, tids):
    nv = vp.shape[0]
    h, w = tg.shape[1], tg.shape[2]
    t = cls(p.shape[0], sh_degree=deg, params=p)
    t.set_targets(tg)
    t.set_views(vp, vpi, tids)
    img = torch.zeros((nv, h, w, 4), device="cuda")
    t.forward(out=img)
    l3 = t.loss()
    t.backward()
    st = t.read_state()
    return t, img.cpu().numpy(), l3, st


CASES = [
    (1024, 64, 64, 0, ((0.0, 0.0, 4.0),), -4.0),
    (3000, 96, 80, 3, ((0.0, 0.0, 4.0), (3.0, 1.0, 2.5)), -3.5),
    (20000, 256, 256, 0, ((0.0, 0.0, 4.0),), -4.0),
]


@pytest.mark.parametrize("n,w,h,deg,eyes,lsm", CASES)
def test_forward_loss_backward_match_oracle(trainer_cls, n, w, h, deg, eyes, lsm):
    p = gs_scene(n, 11 + deg, deg=deg, log_scale_mean=lsm)
    vp, vpi, views = gs_views(w, h, eyes)
    nv = len(eyes)
    tg = gs_targets(nv + 1, w, h, 5)
    tids = np.arange(nv, dtype=np.uint32)[::-1].copy()  # views map to targets out of order
    t, img, l3, st = run_gpu(trainer_cls, p, deg, vp, vpi, tg, tids)
    rimg, rnc = orc.gs_forward(p, deg, views, w, h)
    np.testing.assert_allclose(img, rimg, atol=1e-5, rtol=0)
    rl3, rdimg = orc.gs_loss(rimg, tg, tids)
    # loss and mean L1 to 1e-5 relative; mean SSIM (near 0 for unrelated
    # images) to 2e-5 absolute: its variance terms E[x^2] - mu^2 cancel, and
    # the separable convolutions round differently with FMA on the device
    np.testing.assert_allclose(l3[:2], rl3[:2], rtol=1e-5, atol=1e-7)
    assert abs(l3[2] - rl3[2]) < 2e-5, (l3, rl3)
    img2, dimg = t.read_image()
    np.testing.assert_array_equal(img2, img)
    np.testing.assert_allclose(dimg[..., :3], rdimg[..., :3], atol=1e-6, rtol=1e-4)
    rg, radc = orc.gs_backward(p, deg, views, w, h, rimg, rnc, rdimg, with_adc=True)
    # ADC statistic: views that saw each Gaussian exact, gradient norms 1e-4 relative (L2)
    np.testing.assert_array_equal(st["adc_denom"], radc[:, 1])
    an, bn = st["adc_grad"].astype(np.float64), radc[:, 0].astype(np.float64)
    assert np.linalg.norm(an - bn) / np.linalg.norm(bn) < 1e-4
    g = st["grads"]
    used = np.r_[0:11, 12:12 + 3 * (deg + 1) ** 2]
    a, b = g[:, used].astype(np.float64), rg[:, used].astype(np.float64)
    rel_l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel_l2 < 1e-4, rel_l2
    scale = np.abs(b).max(axis=0, keepdims=True)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * scale)
    assert np.quantile(rel, 0.99) < 1e-3, np.quantile(rel, 0.99)
    assert t.stats()["pairs"] > 0


def test_per_view_accumulation_matches_batched(trainer_cls):
    """The plain per-view trainer's accumulated gradient (one launch per view)
    equals the batched multi-view gradient; so do the loss and ADC statistic."""
    n, w, h, deg = 4000, 96, 96, 1
    p = gs_scene(n, 6, deg=deg, log_scale_mean=-3.6)
    eyes = ((0.0, 0.0, 4.0), (2.8, 0.0, 2.8), (0.0, 2.8, 2.8))
    vp, vpi, views = gs_views(w, h, eyes)
    tg = gs_targets(4, w, h, 12)
    tids = np.array([3, 1, 0], np.uint32)
    t, img, l3, st = run_gpu(trainer_cls, p, deg, vp, vpi, tg, tids)
    u = trainer_cls(n, sh_degree=deg, params=p)
    u.set_targets(tg)
    total = 0.0
    for k in range(3):
        u.set_accumulate(k > 0, 3)
        u.set_views(vp[k:k + 1], vpi[k:k + 1], tids[k:k + 1])
        u.forward()
        total += u.loss()[0]
        u.backward()
    su = u.read_state()
    assert abs(total - l3[0]) < 1e-5 * abs(l3[0])
    a, b = su["grads"].astype(np.float64), st["grads"].astype(np.float64)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
    np.testing.assert_array_equal(su["adc_denom"], st["adc_denom"])
    np.testing.assert_allclose(su["adc_grad"], st["adc_grad"], rtol=1e-4, atol=1e-9)
    # and the whole per-view step is one Adam update of that gradient
    u2 = trainer_cls(n, sh_degree=deg, params=p)
    u2.set_targets(tg)
    u2.train_step_per_view(vp, vpi, tids)
    t.adam()
    # Adam's first update is ~ lr * sign(g): entries whose gradient is summed
    # to ~0 in another atomic order may flip, so compare all but a few
    close = np.isclose(u2.read_state()["params"], t.read_state()["params"], rtol=1e-5, atol=1e-6)
    assert close.mean() > 0.999, close.mean()


def test_gradients_match_fp64_central_differences(trainer_cls):
    """Small-case check: 1024 Gaussians, 64x64, L1 + D-SSIM loss, CUDA
    gradients against FP64 central differences (h = 1e-4 relative)."""
    n, w, h, deg = 1024, 64, 64, 0
    p = gs_scene(n, 2, deg=deg, log_scale_mean=-3.5)
    vp, vpi, views = gs_views(w, h)
    tg = gs_targets(1, w, h, 3)
    tids = np.zeros(1, np.uint32)
    t, img, l3, st = run_gpu(trainer_cls, p, deg, vp, vpi, tg, tids)
    g = st["grads"]
    rng = np.random.default_rng(1)
    touched = np.nonzero(np.abs(g[:, 0]) > 0)[0]
    gi = rng.choice(touched, min(40, len(touched)), replace=False)
    fields = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14]
    pidx = np.array([i * 64 + f for i in gi for f in fields], np.uint32)
    cd = orc.gs_loss_cd(p, deg, views, w, h, tg, tids, pidx)
    an = g.reshape(-1)[pidx].astype(np.float64)
    rel = np.abs(an - cd) / np.maximum(np.abs(cd), 1e-3 * np.abs(cd).max())
    assert np.median(rel) < 1e-4, np.median(rel)
    assert np.quantile(rel, 0.95) < 1e-3, np.quantile(rel, 0.95)


def test_adam_matches_oracle(trainer_cls):
    n, w, h, deg = 2000, 64, 48, 3
    p = gs_scene(n, 4, deg=deg, log_scale_mean=-3.5)
    vp, vpi, views = gs_views(w, h, ((0.0, 0.0, 4.0), (0.0, 3.0, 2.5)))
    tg = gs_targets(2, w, h, 9)
    tids = np.arange(2, dtype=np.uint32)
    t = trainer_cls(n, sh_degree=deg, params=p)
    t.set_targets(tg)
    t.set_views(vp, vpi, tids)
    for _ in range(3):
        t.train_step()
    s0 = t.read_state()
    t.forward()
    t.loss()
    t.backward()
    g = t.read_state()["grads"]
    t.adam()
    s1 = t.read_state()
    pp, mm, vv = s0["params"].copy(), s0["adam_m"].copy(), s0["adam_v"].copy()
    orc.gs_adam(pp, g, mm, vv, 4, t.LR_DEFAULT)
    np.testing.assert_allclose(s1["adam_m"], mm, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(s1["adam_v"], vv, rtol=1e-6, atol=1e-18)
    np.testing.assert_allclose(s1["params"], pp, rtol=1e-6, atol=1e-7)


def test_training_reduces_loss(trainer_cls):
    """Fit a student to a teacher's renders: the loss must drop."""
    n, w, h, deg = 4000, 96, 96, 1
    teacher = gs_scene(n, 21, deg=deg, log_scale_mean=-3.2)
    eyes = ((0.0, 0.0, 4.0), (4.0, 0.0, 0.5), (0.0, 4.0, 0.5), (-3.0, -1.0, 2.5))
    vp, vpi, views = gs_views(w, h, eyes)
    tgt_img, _ = orc.gs_forward(teacher, deg, views, w, h)
    tg = tgt_img.copy()
    tg[..., 3] = 1.0
    student = gs_scene(n, 22, deg=deg, log_scale_mean=-3.2)
    t = trainer_cls(n, sh_degree=deg, params=student)
    t.set_targets(tg)
    t.set_views(vp, vpi, np.arange(4, dtype=np.uint32))
    first = t.train_step(read_loss=True)[0]
    for _ in range(150):
        last = t.train_step(read_loss=True)[0]
    assert last < 0.7 * first, (first, last)


def test_graph_mode_matches_eager_and_recovers_from_overflow(trainer_cls):
    """The captured train step equals the eager one (up to the order of float
    atomics in the backward); a replay whose pairs overflow the captured
    capacity skips its update and the next call recaptures."""
    n, w, h, deg = 3000, 96, 80, 2
    p = gs_scene(n, 40, deg=deg, log_scale_mean=-3.5)
    eyes = ((0.0, 0.0, 4.0), (3.0, 1.0, 2.5))
    vp, vpi, _ = gs_views(w, h, eyes)
    tg = gs_targets(2, w, h, 41)
    runs = []
    for graph in (False, True):
        t = trainer_cls(n, sh_degree=deg, params=p)
        t.set_targets(tg)
        t.set_views(vp, vpi, np.arange(2, dtype=np.uint32))
        t.set_graph(graph)
        losses = [t.train_step(read_loss=True)[0] for _ in range(6)]
        runs.append((t.read_state()["params"], losses, t))
    np.testing.assert_allclose(runs[1][1], runs[0][1], rtol=1e-4)
    np.testing.assert_allclose(runs[1][0], runs[0][0], rtol=1e-3, atol=1e-5)
    t = runs[1][2]
    assert t.stats()["skipped_steps"] == 0
    # much larger Gaussians: 3x the pairs with the same step shape
    big = t.read_state()["params"].copy()
    big[:, 3:6] += 1.5
    t.write_params(big)
    before = t.read_state()["params"].copy()
    t.train_step()                       # replay: overflows, update skipped
    after = t.read_state()["params"]
    np.testing.assert_array_equal(after, before)
    t.train_step()                       # detects the skip, eager step + recapture
    assert t.stats()["skipped_steps"] == 1
    t.train_step()                       # replay of the new graph
    assert not np.array_equal(t.read_state()["params"], before)


def test_deterministic_mode_is_bit_reproducible(trainer_cls, tmp_path):
    """The small case (1024 Gaussians, 64x64) and a larger multi-view case:
    the two-pass backward gives bit-identical gradients run to run, agrees
    with the atomic reduction and the FP64 central differences, and a
    checkpointed run resumes bit-exactly."""
    for n, w, h, deg, eyes in ((1024, 64, 64, 0, ((0.0, 0.0, 4.0),)),
                               (6000, 128, 96, 2, ((0.0, 0.0, 4.0), (2.5, 1.0, 3.0), (-3.0, 0.5, 2.0)))):
        p = gs_scene(n, 50 + deg, deg=deg, log_scale_mean=-3.5)
        vp, vpi, views = gs_views(w, h, eyes)
        nv = len(eyes)
        tg = gs_targets(nv, w, h, 51)
        tids = np.arange(nv, dtype=np.uint32)
        grads = []
        for det in (True, True, False):
            t = trainer_cls(n, sh_degree=deg, params=p)
            t.set_deterministic(det)
            t.set_targets(tg)
            t.set_views(vp, vpi, tids)
            t.forward()
            t.loss()
            t.backward()
            st = t.read_state()
            grads.append((st["grads"], st["adc_grad"]))
            if det:
                t.backward()  # a second backward of the same forward: same bits
                np.testing.assert_array_equal(t.read_state()["grads"], st["grads"])
        np.testing.assert_array_equal(grads[0][0], grads[1][0])
        np.testing.assert_array_equal(grads[0][1], grads[1][1])
        a, b = grads[0][0].astype(np.float64), grads[2][0].astype(np.float64)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
    # 1024 Gaussians at 64x64: deterministic gradients against FP64 central differences
    n, w, h = 1024, 64, 64
    p = gs_scene(n, 2, deg=0, log_scale_mean=-3.5)
    vp, vpi, views = gs_views(w, h)
    tg = gs_targets(1, w, h, 3)
    t = trainer_cls(n, sh_degree=0, params=p)
    t.set_deterministic(True)
    t.set_targets(tg)
    t.set_views(vp, vpi)
    t.forward()
    t.loss()
    t.backward()
    g = t.read_state()["grads"]
    rng = np.random.default_rng(4)
    touched = np.nonzero(np.abs(g[:, 0]) > 0)[0]
    gi = rng.choice(touched, min(30, len(touched)), replace=False)
    pidx = np.array([i * 64 + f for i in gi for f in (0, 1, 2, 3, 4, 5, 6, 10, 12)], np.uint32)
    cd = orc.gs_loss_cd(p, 0, views, w, h, tg, np.zeros(1, np.uint32), pidx)
    an = g.reshape(-1)[pidx].astype(np.float64)
    rel = np.abs(an - cd) / np.maximum(np.abs(cd), 1e-3 * np.abs(cd).max())
    assert np.median(rel) < 1e-4, np.median(rel)
    # graph-captured training is reproducible and resumes bit-exactly
    runs = []
    for _ in range(2):
        u = trainer_cls(n, sh_degree=0, params=p)
        u.set_deterministic(True)
        u.set_graph(True)
        u.set_targets(tg)
        u.set_views(vp, vpi)
        for _ in range(8):
            u.train_step()
        runs.append(u)
    s0, s1 = runs[0].read_state(), runs[1].read_state()
    np.testing.assert_array_equal(s0["params"], s1["params"])
    path = tmp_path / "det.bin"
    runs[0].save(path)
    for _ in range(4):
        runs[0].train_step()
    r = trainer_cls(n, sh_degree=0)
    r.load(path)
    r.set_deterministic(True)
    r.set_graph(True)
    r.set_targets(tg)
    r.set_views(vp, vpi)
    for _ in range(4):
        r.train_step()
    np.testing.assert_array_equal(r.read_state()["params"], runs[0].read_state()["params"])
    np.testing.assert_array_equal(r.read_state()["adam_v"], runs[0].read_state()["adam_v"])


def test_raster_variants_agree_and_autotune(trainer_cls, tmp_path):
    """Forward images agree across tile sizes (8, 16, 32) and the raster
    variants of both forms (one CTA per tile; persistent warp-specialised)
    and 1 / 2 / 4 pixels per thread to 1e-6 (the compiler may fuse
    multiply-adds differently in each instantiation; each pixel composites
    the same Gaussians in the same depth order whatever the tile); backward
    gradients to 1e-5 relative L2, also with the forward and backward in
    different forms; both match the oracle; the autotuner times every
    variant of every tile, picks a valid one and reuses its cached choice."""
    n, w, h, deg = 5000, 112, 96, 2
    p = gs_scene(n, 61, deg=deg, log_scale_mean=-3.4)
    eyes = ((0.0, 0.0, 4.0), (2.5, 1.0, 3.0))
    vp, vpi, views = gs_views(w, h, eyes)
    tg = gs_targets(2, w, h, 62)
    t = trainer_cls(n, sh_degree=deg, params=p)
    t.set_targets(tg)
    t.set_views(vp, vpi)
    imgs, grads, ncs = {}, {}, {}
    variants = [(16, 0) + va for va in t.VARIANTS] + [(16, 2) + va for va in t.VARIANTS]
    variants += [(tile, 1) + va for tile, vs in t.PERSISTENT_VARIANTS.items() for va in vs]
    for va in variants:
        t.set_tile(va[0])
        t.set_raster(va[1:], va[1:])
        t.forward()
        t.loss()
        t.backward()
        imgs[va] = t.read_image(with_grad=False)[0]
        grads[va] = t.read_state()["grads"].astype(np.float64)
        if va[0] == 16:
            # the persistent backward after a grid forward (and the reverse): the
            # per-tile last contributors both forms write drive either backward
            other = (0,) + t.VARIANTS[1] if va[1] != 0 else (1,) + t.PERSISTENT_VARIANTS[16][1]
            t.set_raster(other, va[1:])
            t.forward()
            t.loss()
            t.backward()
            ncs[va] = t.read_state()["grads"].astype(np.float64)
    base = (16, 0, 1, 256)
    for va in variants[1:]:
        np.testing.assert_allclose(imgs[va], imgs[base], atol=1e-6, rtol=0)
        assert np.linalg.norm(grads[va] - grads[base]) / np.linalg.norm(grads[base]) < 1e-5, va
    for va, g in ncs.items():
        assert np.linalg.norm(g - grads[base]) / np.linalg.norm(grads[base]) < 1e-5, va
    rimg, rnc = orc.gs_forward(p, deg, views, w, h)
    np.testing.assert_allclose(imgs[16, 0, 4, 128], rimg, atol=1e-5, rtol=0)
    np.testing.assert_allclose(imgs[16, 1, 2, 128], rimg, atol=1e-5, rtol=0)
    np.testing.assert_allclose(imgs[32, 1, 4, 128], rimg, atol=1e-5, rtol=0)
    np.testing.assert_allclose(imgs[8, 1, 1, 64], rimg, atol=1e-5, rtol=0)
    t.set_tile(16)
    from nprush_b200._lib import NpsError
    with pytest.raises(NpsError):
        t.set_variant(1, 1, 512, 512)
    cache = tmp_path / "autotune.txt"
    r = t.autotune(cache)
    for pas in ("fwd", "bwd"):
        table = t.PERSISTENT_VARIANTS[r["tile"]] if r[f"{pas}_form"] == 1 else t.VARIANTS
        assert (r[f"{pas}_ppt"], r[f"{pas}_stage"]) in table
        assert r[f"{pas}_form"] == 1 or r["tile"] == 16
    assert not r["cached"]
    for tile, row in r["per_tile"].items():
        assert row["binning_ms"] > 0
        served = [(v[0] != 1 and tile == 16) or (v[0] == 1 and v[1:] in t.PERSISTENT_VARIANTS[tile])
                  for v in t.TUNE_VARIANTS]
        assert [x > 0 for x in row["fwd_ms"]] == served and [x > 0 for x in row["bwd_ms"]] == served, (tile, row)
    r2 = t.autotune(cache)
    keys = ("tile", "fwd_form", "fwd_ppt", "fwd_stage", "bwd_form", "bwd_ppt", "bwd_stage")
    assert r2["cached"] and [r2[k] for k in keys] == [r[k] for k in keys]
    # the tuned trainer still trains
    t.set_graph(True)
    l0 = t.train_step(read_loss=True)[0]
    for _ in range(5):
        t.train_step()
    assert t.train_step(read_loss=True)[0] < l0


def test_upload_targets_matches_set_targets(trainer_cls):
    """Targets uploaded by ids from page-locked host memory (side stream) give
    the same step as the same images set directly; an upload queued after a
    step does not change that step."""
    n, w, h = 3000, 64, 48
    p = gs_scene(n, 71, deg=1, log_scale_mean=-3.4)
    vp, vpi, _ = gs_views(w, h, ((0.0, 0.0, 4.0), (2.5, 1.0, 3.0)))
    allt = torch.from_numpy(gs_targets(5, w, h, 72)).pin_memory()
    hs = allt.numpy()
    ids = np.array([3, 1], np.uint32)
    # deterministic mode: the comparisons below are bit for bit
    a = trainer_cls(n, sh_degree=1, params=p)
    a.set_deterministic(True)
    a.set_targets(hs[ids])
    a.set_views(vp, vpi)
    la = a.train_step(read_loss=True)
    b = trainer_cls(n, sh_degree=1, params=p)
    b.set_deterministic(True)
    b.upload_targets(hs, ids)
    b.set_views(vp, vpi)
    b.train_step()
    b.upload_targets(hs, np.array([0, 4], np.uint32))  # queued behind the step
    lb = b.read_loss()
    assert la == lb
    np.testing.assert_array_equal(a.read_state()["params"], b.read_state()["params"])
    b.train_step()
    c = trainer_cls(n, sh_degree=1, params=p)
    c.set_deterministic(True)
    c.set_targets(hs[ids])
    c.set_views(vp, vpi)
    c.train_step()
    c.set_targets(hs[[0, 4]])
    assert c.train_step(read_loss=True) == b.read_loss()


def test_sharded_trainer_single_rank_nccl(trainer_cls):
    """The view-sharded trainer on a one-rank NCCL group: the gradient and ADC
    buffers are all-reduced in place through tensors aliasing the library's
    device memory; the result equals the plain step bit for bit
    (deterministic mode)."""
    import os

    import torch.distributed as dist

    from nprush_b200.distributed import ShardedTrainer, device_tensor
    n, w, h = 3000, 64, 48
    p = gs_scene(n, 81, deg=1, log_scale_mean=-3.4)
    vp, vpi, _ = gs_views(w, h, ((0.0, 0.0, 4.0), (2.5, 1.0, 3.0), (-2.0, 1.0, 3.2)))
    tg = gs_targets(3, w, h, 82)
    ids = np.arange(3, dtype=np.uint32)
    a = trainer_cls(n, sh_degree=1, params=p)
    a.set_deterministic(True)
    a.set_targets(tg)
    a.set_views(vp, vpi, ids)
    for _ in range(3):
        a.train_step()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{29400 + os.getpid() % 500}", rank=0,
                            world_size=1)
    try:
        b = trainer_cls(n, sh_degree=1, params=p)
        b.set_deterministic(True)
        b.set_targets(tg)
        st = ShardedTrainer(b)
        for _ in range(3):
            st.train_step(vp, vpi, ids)
        np.testing.assert_array_equal(b.read_state()["params"], a.read_state()["params"])
        g = device_tensor(b.buffers()["grads"], n * 64, 0)
        assert g.shape[0] == n * 64 and g.is_cuda
        c = st.adc(grad_thresh=1e-6)
        assert c["after"] > 0
    finally:
        dist.destroy_process_group()


def test_sort_lookback_timeout_is_reported(trainer_cls):
    """The onesweep sorts' bounded look-back, made to run out on a normal
    input (tile 2 of each sort treated as never published, 1000 polls): the
    train step raises NPS_ERR_TIMEOUT, the parameters are not updated, and once
    the guard is back to normal the trainer continues exactly as a fresh one
    (deterministic mode)."""
    from nprush_b200._lib import NpsError
    n, w, h = 20000, 256, 256
    p = gs_scene(n, 101, deg=0, log_scale_mean=-3.5)
    vp, vpi, _ = gs_views(w, h)
    tg = gs_targets(1, w, h, 102)
    runs = []
    for stall in (True, False):
        t = trainer_cls(n, sh_degree=0, params=p)
        t.set_deterministic(True)
        t.set_targets(tg)
        t.set_views(vp, vpi)
        if stall:
            t.set_sort_guard(1000, 2)
            with pytest.raises(NpsError) as e:
                t.train_step()
            assert e.value.code == -5 and t.stats()["staging_timeouts"] > 0
            np.testing.assert_array_equal(t.read_state()["params"], p)
            t.set_sort_guard()
        for _ in range(3):
            t.train_step()
        runs.append(t.read_state()["params"])
    np.testing.assert_array_equal(runs[0], runs[1])
