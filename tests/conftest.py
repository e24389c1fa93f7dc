import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def L():
    from clspmv_b200 import capi
    return capi.lib()


@pytest.fixture(scope="session")
def ref():
    from tests import _oracle
    r = _oracle.ref_lib()
    if r is None:
        pytest.skip("reference oracle oracle/_ref/libclspmv_ref.so not built")
    return r


@pytest.fixture(scope="session")
def orc():
    from tests import _oracle
    return _oracle.oracle_lib()
