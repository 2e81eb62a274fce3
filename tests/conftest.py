import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and the built libsci_cuda.so")


@pytest.fixture(scope="session")
def oracle():
    from tests import _oracle

    return _oracle.port()


@pytest.fixture(scope="session")
def reference():
    from tests import _oracle

    lib = _oracle.reference()
    if lib is None:
        pytest.skip("oracle/_ref/libsci_ref.so is not built (needs the reference sources)")
    return lib


@pytest.fixture(scope="session")
def device():
    from libsci_b200.device import Device

    dev = Device(0)
    yield dev
    dev.close()
