"""The target-preprocessing fixtures (tests/golden/preprocess.npz, outputs of
the reference's own blur / depth-aware blur / splat edge shaders run on the
host) against the numpy restatement in oracle/preprocess.py (1e-5: the
restatement accumulates in double, the shaders in float); when the reference
checkout is present, the shaders are run again and must reproduce the
fixtures bit for bit."""
from pathlib import Path

import numpy as np

import preprocess as pre
from conftest import requires_reference

GOLD = Path(__file__).resolve().parent / "golden" / "preprocess.npz"


def test_restatement_matches_the_fixtures():
    d = np.load(GOLD)
    for k, (dx, dy, r, f) in enumerate(d["blur_cases"]):
        np.testing.assert_allclose(pre.blur(d["color"], (dx, dy), r, f, float(d["blur_sigmas"][k])), d[f"blur{k}"],
                                   atol=1e-5, rtol=0)
    for k, r in enumerate(d["depth_blur_radii"]):
        np.testing.assert_allclose(pre.depth_aware_blur(d["color"], d["depth"], int(r)), d[f"depth_blur{k}"],
                                   atol=1e-5, rtol=0)
    tmin, tmax = d["edge_thresholds"]
    np.testing.assert_allclose(pre.splat_edge(d["depth"], float(tmin), float(tmax)), d["edge"], atol=1e-5, rtol=0)
    assert (d["edge"][..., 0] > 0.5).sum() > 50  # the silhouette is there


@requires_reference
def test_reference_shaders_reproduce_the_fixtures(tmp_path, monkeypatch):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", GOLD.parent / "make_preprocess_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    monkeypatch.setattr(mk, "HERE", tmp_path)
    mk.main()
    a, b = np.load(GOLD), np.load(tmp_path / "preprocess.npz")
    for k in a.files:
        np.testing.assert_array_equal(a[k], b[k])
