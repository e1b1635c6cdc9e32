import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
os.environ.setdefault("FPT_QUIET", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def fpt():
    from falcor_b200 import build
    build.build()
    from falcor_b200 import _ffi
    return _ffi.lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle import ffi
    ffi.build()
    return ffi
