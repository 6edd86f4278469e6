import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (run with -m gpu)")


@pytest.fixture(scope="session")
def engine():
    """The C ABI of the engine, with the CUDA path required."""
    import minhashcuda_b200
    return minhashcuda_b200.capi()
