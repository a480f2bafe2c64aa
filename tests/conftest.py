import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "cube-tracing_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA kernels")


@pytest.fixture(scope="session")
def oracle_lib():
    import pyoracle
    if not pyoracle.available():
        pytest.fail("oracle library not built (make -C oracle)")
    return pyoracle
