import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def gf():
    import __graft_entry__
    return __graft_entry__.import_package()


@pytest.fixture(scope="session")
def refrun():
    from oracle import refrun as rr
    if not rr.available():
        pytest.skip("oracle binary not built (make -C oracle)")
    return rr
