"""C-ABI checks that need no GPU: the library loads and exports every entry
point include/nprush.h declares; calls fail cleanly (status + message)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = "\n".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nps_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from nprush_b200 import build
    build.build()
    return ctypes.CDLL(str(build.OUT))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "nps_create" in syms and "nps_splat_opt_dispatch" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_every_symbol():
    from nprush_b200 import _lib
    known = set(_lib.SIGNATURES) | set(_lib._RET)
    missing = [s for s in declared_symbols() if s not in known]
    assert not missing, f"no ctypes signature for: {missing}"


def test_version_and_error_strings(lib):
    lib.nps_version.restype = ctypes.c_char_p
    lib.nps_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.nps_version()
    assert isinstance(lib.nps_last_error(), bytes)


def test_null_arguments_are_rejected(lib):
    # argument checks happen before any CUDA call, so this runs without a GPU
    assert lib.nps_create(0, None) == -1
    assert lib.nps_splat_opt_create(None, 0, None) == -1
    lib.nps_last_error.restype = ctypes.c_char_p
    assert b"bad arguments" in lib.nps_last_error()
    assert lib.nps_destroy(None) == 0
