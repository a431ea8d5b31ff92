"""The onesweep radix sort (nps_sort_pairs) against numpy's stable sort, at
the sizes the trainer sorts (the benchmark step's 13.7M tile keys and 1.6M
depth keys) and at the edges (one pair, one tile, a partial last tile, all
keys equal, every digit present); and its bounded look-back: a tile whose
status is never published makes the look-back give up with NPS_ERR_TIMEOUT
(writing nothing outside the buffers), after which the context is usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def lib():
    from nprush_b200 import _lib, build
    build.build()
    return _lib


def sort_on_device(lib, keys, vals, bits, spin_limit=0, stall=0xFFFFFFFF):
    k = torch.from_numpy(keys.view(np.int32)).cuda()
    v = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    rc = lib.load().nps_sort_pairs(lib.context(0), ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                   len(keys), bits, spin_limit, stall)
    return rc, k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


CASES = [
    ("tile keys of the benchmark step", 13_753_049, 15),
    ("depth keys of the benchmark step", 1_600_000, 32),
    ("one pair", 1, 32),
    ("one tile", 3072, 8),
    ("a partial last tile", 3 * 3072 + 17, 20),
    ("all keys equal", 50_000, 32),
    ("every digit present", 256 * 64, 8),
]


@pytest.mark.parametrize("what,n,bits", CASES, ids=[c[0] for c in CASES])
def test_sort_matches_numpy_stable(lib, what, n, bits):
    rng = np.random.default_rng(n)
    if what == "all keys equal":
        keys = np.full(n, 0xDEADBEEF, np.uint32)
    elif what == "every digit present":
        keys = np.repeat(np.arange(256, dtype=np.uint32), 64)[rng.permutation(n)]
    elif bits == 32:
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] = keys[n // 3: 2 * (n // 3)]  # repeated keys: stability matters
    else:
        keys = rng.integers(0, 2 ** bits, n, dtype=np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    rc, k, v = sort_on_device(lib, keys, vals, bits)
    assert rc == 0, lib.load().nps_last_error()
    mask = np.uint32(0xFFFFFFFF if bits == 32 else (1 << bits) - 1)
    order = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(v, vals[order])
    np.testing.assert_array_equal(k, keys[order])


def test_lookback_gives_up_on_a_stalled_tile(lib):
    """Tile 2's status is treated as never published and the look-back may
    poll it 1000 times: the sort reports NPS_ERR_TIMEOUT, writes nothing
    outside its buffers (guard words around them stay untouched: output
    positions are clamped to the key count), and the next sort on the same
    context is correct."""
    n, bits, guard = 40 * 3072, 16, 4096
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 2 ** bits, n, dtype=np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    kbuf = torch.full((n + 2 * guard,), -7, dtype=torch.int32, device="cuda")
    vbuf = torch.full((n + 2 * guard,), -9, dtype=torch.int32, device="cuda")
    kbuf[guard:guard + n] = torch.from_numpy(keys.view(np.int32)).cuda()
    vbuf[guard:guard + n] = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    L = lib.load()
    rc = L.nps_sort_pairs(lib.context(0), ctypes.c_void_p(kbuf.data_ptr() + 4 * guard),
                          ctypes.c_void_p(vbuf.data_ptr() + 4 * guard), n, bits, 1000, 2)
    assert rc == -5  # NPS_ERR_TIMEOUT
    assert b"gave up" in L.nps_last_error()
    kb, vb = kbuf.cpu().numpy(), vbuf.cpu().numpy()
    assert (kb[:guard] == -7).all() and (kb[guard + n:] == -7).all()
    assert (vb[:guard] == -9).all() and (vb[guard + n:] == -9).all()
    rc, k, v = sort_on_device(lib, keys, vals, bits)
    assert rc == 0
    np.testing.assert_array_equal(v, np.argsort(keys, kind="stable").astype(np.uint32))
