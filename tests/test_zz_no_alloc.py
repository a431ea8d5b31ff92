"""The allocation-free ADC entry point (nps_splat_adc_noalloc) against the
allocating one (nps_splat_opt_adc), through the C ABI on the GPU.

nps_splat_adc_noalloc exists for callers that cannot let the library allocate
device memory (an application whose own arena owns the device-memory budget,
or one sharing the GPU with latency-critical work where cudaMalloc / cudaFree
may synchronise the device).  Its scratch lives in a fixed array compiled into
the library, reused by every call.  Both entry points run the same kernel, so
the results must be identical (the ADC tolerance of the other tests is exact
apart from the sinf clone jitter, which is the same code here); two calls in a
row check that the kept scratch contents of one call do not leak into the next.
This file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from scenes import splat_scene  # noqa: E402


def state(n, seed, dead_fraction=0.35):
    rng = np.random.default_rng(seed)
    s = splat_scene(n, seed)
    dead = rng.random(n) < dead_fraction
    s[dead, 7] = 0.0
    s[::7, 3] = 0.002; s[::7, 12] = 0.002; s[::7, 15] = 0.002
    ga = (rng.random(n) * 4e-3).astype(np.float32)
    m = rng.normal(0, 1e-3, (n, 16)).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-5, (n, 16))).astype(np.float32)
    return s, m, v, ga


def check_against_allocating(n, seed, dead_fraction=0.35):
    from nprush_b200 import _lib, build
    build.build()
    from nprush_b200.splat import GpuSplatOptimizerManager
    lib = _lib.load()
    s, m, v, ga = state(n, seed, dead_fraction)
    ref = GpuSplatOptimizerManager(n, init=s)
    dev = [torch.from_numpy(x.copy()).cuda() for x in (s, m, v, ga)]
    stream = torch.cuda.current_stream()
    for call, t in ((0, 50.0), (1, 75.0)):
        if call == 1:
            # the first call filled every dead slot: kill a third of the splats
            # and draw fresh accumulators, identically on both sides
            rng = np.random.default_rng(seed + 1)
            st = ref.read_state()
            s2 = st["splats"].copy()
            s2[rng.random(n) < 0.33, 7] = 0.0
            ga2 = (rng.random(n) * 4e-3).astype(np.float32)
            ref.write_params(s2)
            ref.write_state(st["adam_m"], st["adam_v"], t, ga2)
            dev[0].copy_(torch.from_numpy(s2))
            dev[3].copy_(torch.from_numpy(ga2))
        else:
            ref.write_state(m, v, t, ga)
        ref.adc()
        want = ref.read_state()
        clones = ctypes.c_uint32(0)
        rc = lib.nps_splat_adc_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), dev[3].data_ptr(),
                                       n, ctypes.c_float(t), ctypes.c_void_p(stream.cuda_stream),
                                       ctypes.byref(clones))
        assert rc == 0, lib.nps_last_error()
        assert clones.value == ref.stats()["adc_clones"] > 0
        got = [x.cpu().numpy() for x in dev]
        np.testing.assert_array_equal(got[0], want["splats"])
        np.testing.assert_array_equal(got[1], want["adam_m"])
        np.testing.assert_array_equal(got[2], want["adam_v"])
        np.testing.assert_array_equal(got[3], want["grad_accum"])


def test_noalloc_adc_matches_allocating_entry_point():
    check_against_allocating(20000, 31)


def test_noalloc_adc_at_its_capacity():
    """At the scratch's limit of 262144 splats with most of them dead, the
    dead-slot list fills nearly the whole array up to the result words."""
    check_against_allocating(262144, 33, dead_fraction=0.97)


def test_noalloc_adc_rejects_misaligned_buffers():
    """Offset views that break the kernel's 16-byte (records) or 4-byte
    (accumulators) alignment are rejected on the host, before any launch."""
    from nprush_b200 import _lib
    lib = _lib.load()
    buf = torch.zeros(4096, device="cuda")
    p = buf.data_ptr()
    for args in ((p + 4, p, p, p), (p, p + 8, p, p), (p, p, p + 12, p), (p, p, p, p + 2)):
        rc = lib.nps_splat_adc_noalloc(*args, 16, ctypes.c_float(0.0), None, None)
        assert rc == -1  # NPS_ERR_INVALID
        assert b"aligned" in lib.nps_last_error()


def test_noalloc_adc_rejects_sizes_beyond_its_scratch():
    from nprush_b200 import _lib
    lib = _lib.load()
    buf = torch.zeros(16, device="cuda")
    p = buf.data_ptr()
    rc = lib.nps_splat_adc_noalloc(p, p, p, p, 262145, ctypes.c_float(0.0), None, None)
    assert rc == -4  # NPS_ERR_CAPACITY
    assert b"exceed the fixed scratch" in lib.nps_last_error()
