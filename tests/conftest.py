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


@pytest.fixture(scope="session")
def R():
    """The reference's own FD MEX sources built into oracle/_ref (make -C oracle ref).  They
    are built where the reference tree is present and travel with the repository; a host
    that has neither the built files nor the tree skips the tests that need them."""
    from oracle import swd_ref
    if not swd_ref.available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=False, capture_output=True)
    if not swd_ref.available():
        pytest.skip("oracle/_ref is not built and the reference sources are not here")
    return swd_ref
