"""bench.py's reference arms on the CPU: one JSON line each, with the keys the
measurement contract asks for (the GPU arms run on the GPU only)."""
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
