import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def tb():
    import taucs_b200
    taucs_b200.lib()
    return taucs_b200


@pytest.fixture(scope="session")
def ref():
    from oracle.bindings import Ref, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref/libtaucs_ref.so not built")
    return Ref(threads=1)


@pytest.fixture(scope="session")
def port():
    from oracle.bindings import Port, port_available
    if not port_available():
        pytest.skip("oracle/_ref/liboracle.so not built")
    return Port()
