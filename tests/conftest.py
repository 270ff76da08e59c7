import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")


@pytest.fixture(scope="session")
def hp():
    """The CUDA library binding; skips nothing -- a missing .so is an error."""
    import quadprec_b200 as hp_mod

    return hp_mod


@pytest.fixture(scope="session")
def gpu(hp):
    assert hp.device_ok(), "no sm_100 CUDA device visible"
    return hp
