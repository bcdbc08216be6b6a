import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (the pass itself); parity against the CPU oracle")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """The native library and the oracle, built in-tree if a source is newer (no GPU needed to build)."""
    from threert_b200 import build
    import oracle
    build.build()
    oracle.build()


@pytest.fixture(scope="session")
def gpu():
    from threert_b200 import Gpu
    g = Gpu(int(os.environ.get("TRT_TEST_DEVICE", "0")))
    yield g
    g.close()
