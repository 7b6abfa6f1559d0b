import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running (full-size workloads)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.binding import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.binding import Reference
    if not Reference.available():
        pytest.skip("reference library oracle/_ref/libu3dref.so is not built (reference sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def u3dg():
    """The product library's Python API; fails loudly if libu3dg.so is missing."""
    from univeral_3d_reconstruction_system_b200 import api, _lib
    _lib.load()
    return api


@pytest.fixture(scope="session")
def cpu_threads():
    return max(1, min(os.cpu_count() or 1, 16))
