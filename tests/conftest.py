import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libswd.so kernels)")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Build the CPU oracle library if it is missing (it is only a checker)."""
    so = os.path.join(ROOT, "oracle", "_build", "libswd_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    yield


@pytest.fixture(scope="session")
def O():
    from oracle import swd_oracle
    return swd_oracle
