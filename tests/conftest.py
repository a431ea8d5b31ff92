import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "reference: needs the reference checkout to build oracle/_ref")


def reference_available() -> bool:
    from build_ref import reference_available as ra
    return ra()


def _reference_root() -> Path:
    from build_ref import reference_root
    return reference_root()


requires_reference = pytest.mark.skipif(
    not (_reference_root() / "src/lib/gpu").is_dir(),
    reason="reference checkout not present (oracle/_ref cannot be built)")
