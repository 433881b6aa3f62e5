import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built_artifacts():
    """Build the oracle (the checker) and the CUDA library if missing."""
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATH):
        O.build()
    from hnsw_rabitq_b200 import build as B
    if B.stale():
        try:
            B.build()
        except Exception:  # no nvcc on this machine: tests that need the library fail loudly themselves
            pass
    yield
