import os
import sys

import pytest

TESTS_DIR = os.path.dirname(os.path.abspath(__file__))
if TESTS_DIR not in sys.path:
    sys.path.insert(0, TESTS_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU-only test")


@pytest.fixture(scope="session")
def oracle():
    from dms_ctypes import Oracle
    o = Oracle()
    yield o
    o.close()


def pytest_sessionstart(session):
    """Build the C oracle if it is missing (gcc only; the reference build is optional)."""
    from dms_ctypes import ORACLE_LIB, REPO
    if not os.path.exists(ORACLE_LIB):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), os.path.join(REPO, "oracle", "liboracle.so")],
                       check=True, stdout=subprocess.DEVNULL)
