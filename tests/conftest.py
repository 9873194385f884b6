import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "svn-export_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def gpu():
    import mhdarcy
    if not mhdarcy.device_available():
        pytest.fail("gpu-marked test run without a CUDA device")
    return True
