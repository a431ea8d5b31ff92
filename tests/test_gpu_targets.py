"""GPU target preprocessing (blur, depth-aware blur, splat edge) against the
reference's own shaders' outputs (tests/golden/preprocess.npz).

Tolerances: stored floats 2e-6 absolute (CUDA's expf / powf against the host
libm's, float sums in the same order); with quantize=True the 8-bit levels are
equal wherever the reference's float is not within 1e-5 of a rounding edge."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLD = Path(__file__).resolve().parent / "golden" / "preprocess.npz"


@pytest.fixture(scope="module")
def tg():
    from nprush_b200 import build
    build.build()
    from nprush_b200 import targets
    return targets


def check(got, want):
    np.testing.assert_allclose(got, want, atol=2e-6, rtol=0)


def check_q(got_q, want_raw):
    want_q = np.rint(np.clip(want_raw, 0, 1) * 255) / 255
    frac = np.clip(want_raw, 0, 1) * 255 - np.floor(np.clip(want_raw, 0, 1) * 255)
    edge = np.abs(frac - 0.5) < 1e-5 * 255
    assert np.all((got_q == want_q) | edge)


def test_blur(tg):
    d = np.load(GOLD)
    src = torch.from_numpy(d["color"]).cuda()
    for k, (dx, dy, r, f) in enumerate(d["blur_cases"]):
        for q in (False, True):
            dst = torch.zeros_like(src)
            tg.blur(src, dst, (int(dx), int(dy)), int(r), float(d["blur_sigmas"][k]), int(f), quantize=q)
            (check_q if q else check)(dst.cpu().numpy(), d[f"blur{k}"])


def test_depth_aware_blur(tg):
    d = np.load(GOLD)
    c, z = torch.from_numpy(d["color"]).cuda(), torch.from_numpy(d["depth"]).cuda()
    for k, r in enumerate(d["depth_blur_radii"]):
        for q in (False, True):
            dst = torch.zeros_like(c)
            tg.depth_aware_blur(c, z, dst, int(r), quantize=q)
            (check_q if q else check)(dst.cpu().numpy(), d[f"depth_blur{k}"])


def test_splat_edge(tg):
    d = np.load(GOLD)
    z = torch.from_numpy(d["depth"]).cuda()
    tmin, tmax = (float(x) for x in d["edge_thresholds"])
    for q in (False, True):
        dst = torch.zeros_like(z)
        tg.splat_edge(z, dst, tmin, tmax, quantize=q)
        (check_q if q else check)(dst.cpu().numpy(), d["edge"])


def test_bad_arguments_are_rejected(tg):
    from nprush_b200._lib import NpsError
    a = torch.zeros((8, 8, 4), device="cuda")
    with pytest.raises(NpsError):
        tg.blur(a, a, (1, 0), 2, 1.0)  # in place
    with pytest.raises(NpsError):
        tg.blur(a, torch.zeros_like(a), (1, 0), 2, 0.0)  # sigma 0


def test_blur_manager_classes(tg):
    """GpuBlurPipelineManager.blur runs the horizontal pass into the temp
    image and the vertical pass into dst, with 8-bit levels between them:
    equal to those two single passes (each pinned to the reference shader by
    test_blur).  The depth-aware manager at radius 3 matches the reference's
    8-bit levels of the fixture."""
    d = np.load(GOLD)
    src = torch.from_numpy(d["color"]).cuda()
    h, w = src.shape[:2]
    temp, dst = torch.zeros_like(src), torch.zeros_like(src)
    tg.GpuBlurPipelineManager().blur(src, dst, temp, w, h, 6, 3.0, is_srgb=True)
    t2, d2 = torch.zeros_like(src), torch.zeros_like(src)
    tg.blur(src, t2, (1, 0), 6, 3.0, tg.SRGB_IN, quantize=True)
    tg.blur(t2, d2, (0, 1), 6, 3.0, tg.SRGB_OUT, quantize=True)
    assert torch.equal(temp, t2) and torch.equal(dst, d2)
    with pytest.raises(ValueError):
        tg.GpuBlurPipelineManager().blur(src, dst, temp, w + 1, h, 6, 3.0)
    z = torch.from_numpy(d["depth"]).cuda()
    k = [int(r) for r in d["depth_blur_radii"]].index(3)
    out = torch.zeros_like(src)
    tg.GpuDepthAwareBlurPipelineManager().blur(src, z, out, w, h, 3)
    check_q(out.cpu().numpy(), d[f"depth_blur{k}"])
