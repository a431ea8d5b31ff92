"""bench.py on the CPU: the reference arms (one JSON line each, with the keys
the measurement contract asks for) and the roofline helpers (the GPU arms run
on the GPU only)."""
import io
import json
import runpy
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def run_bench(*argv):
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    buf = io.StringIO()
    try:
        with redirect_stdout(buf):
            runpy.run_path(str(ROOT / "bench.py"), run_name="__main__")
    finally:
        sys.argv = old
    lines = [l for l in buf.getvalue().splitlines() if l.strip()]
    assert len(lines) == 1, lines
    return json.loads(lines[0])


def test_mesh_raster_reference_arm():
    """The reference's own mesh / envmap stage functions between the restated
    fixed-function steps, timed at two sizes and evaluated at the workload's
    (needs oracle/_ref's mesh build, made from the reference checkout)."""
    if not list((ROOT / "oracle" / "_ref").glob("mesh_n0_*.so")):
        import build_ref
        if not build_ref.reference_available():
            pytest.skip("oracle/_ref has no mesh stages and the reference checkout is absent")
    line = run_bench("--workload", "mesh_raster", "--impl", "reference", "--steps", "1", "--warmup", "3")
    assert line["impl"] == "reference" and line["unit"] == "passes/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and "fitted" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["value"] == line["value"] and line["higher_is_better"] is True


def test_path_trace_reference_arm():
    """The reference's own path_trace.wgsl, translated and run on the host, on
    a bounded sample of the workload (needs oracle/_ref, built from the
    reference checkout)."""
    if not list((ROOT / "oracle" / "_ref").glob("path_trace_n0_*.so")):
        import build_ref
        if not build_ref.reference_available():
            pytest.skip("oracle/_ref has no path tracer and the reference checkout is absent")
    line = run_bench("--workload", "path_trace", "--impl", "reference", "--steps", "1", "--warmup", "3")
    assert line["impl"] == "reference" and line["unit"] == "samples/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "samples/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["higher_is_better"] is True


def _bench_module():
    return runpy.run_path(str(ROOT / "bench.py"), run_name="bench_helpers")


def test_issue_roofline_arithmetic():
    """roofline.issue: the recorded instruction count of the variant that ran,
    scaled by the step's pairs, over the stage time, against 148 SMs x 4
    schedulers x the sampled SM clock; none for variants without a count."""
    b = _bench_module()
    tuned = {"tile": 16, "fwd_form": 2, "fwd_ppt": 2, "fwd_stage": 128, "bwd_form": 2, "bwd_ppt": 2,
             "bwd_stage": 128}
    inst, pairs = b["RASTER_INST"][("raster_bwd", 2, 2, 128)]
    r = b["issue_roofline"]("raster_bwd", tuned, 2 * pairs, 2.0, 1965.0)
    peak = 148 * 4 * 1965.0 * 1e-3
    assert r["bound"] == "issue" and abs(r["peak"] - peak) < 1e-9
    assert abs(r["inst_per_launch"] - 2 * inst) < 1.0
    assert abs(r["achieved"] - 2 * inst / 2e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / peak) < 1e-12
    assert b["issue_roofline"]("raster_bwd", dict(tuned, tile=8), pairs, 1.0, 1965.0) is None
    assert b["issue_roofline"]("raster_bwd", dict(tuned, bwd_ppt=4), pairs, 1.0, 1965.0) is None
    assert b["issue_roofline"]("raster_fwd", None, pairs, 1.0, 1965.0) is None


def test_recorded_counts_are_per_launch_of_the_benchmark_workload():
    """The instruction and traffic constants come from captures of the
    benchmark workload's own pair count (scaled linearly by pairs)."""
    b = _bench_module()
    for (stage, form, ppt, sps), (inst, pairs) in b["RASTER_INST"].items():
        assert stage in ("raster_fwd", "raster_bwd") and inst > pairs > 1_000_000
    assert b["BWD_TRAFFIC_BYTES"] > 0 and b["BWD_TRAFFIC_PAIRS"] > 1_000_000
