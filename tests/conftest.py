import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cybershake-core_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the compiled sm_100a path")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and (when nvcc is present) the library once."""
    import subprocess
    subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    subprocess.run(["make", "-s", "-C", PKG], check=True)
    yield
