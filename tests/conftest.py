import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running GPU case")


def _ensure_built():
    """Build the native libraries when they are missing and a compiler is
    present (here); on a GPU box the prebuilt objects travel with the tree."""
    from flowpsi_b200 import _build
    import oracle.build as ob

    if not _build.LIB.exists():
        _build.build()
    if not ob.LIB.exists():
        ob.build_oracle()
    if not ob.REF_LIB.exists():
        ob.build_ref()


_ensure_built()


def gpu_available() -> bool:
    try:
        from flowpsi_b200 import _native as N

        return bool(N.lib().fpsi_device_available())
    except Exception:
        return False


@pytest.fixture(scope="session")
def need_gpu():
    if not gpu_available():
        pytest.fail("a -m gpu test ran without a CUDA device")
