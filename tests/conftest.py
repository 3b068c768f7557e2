import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_cases.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libnumpp_b200.so")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def oracle():
    from oracle import load_oracle
    return load_oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import load_ref, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present here")
    return load_ref()


@pytest.fixture(scope="session")
def lib():
    """The C ABI on a GPU box: the library must load and see an sm_100 device."""
    from numpp_b200 import _lib
    L = _lib.load()
    assert L.nppb_device_available() == 1, "no sm_100 device visible: " + _lib.last_error()
    return L
