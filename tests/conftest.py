import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and libdvm_cuda.so (run with -m gpu)")


@pytest.fixture(scope="session")
def ctx():
    from dvmpp_b200 import native

    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def port():
    from oracle.pyoracle import Port

    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.pyoracle import Ref, have_ref

    if not have_ref():
        pytest.skip("reference build (oracle/_ref/libdvmref.so) not present")
    return Ref()
