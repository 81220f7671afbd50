import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build(ref=True)
    return Oracle()


@pytest.fixture(scope="session")
def ref(oracle):
    from oracle.oracle import Ref, ref_available
    if not ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    return Ref()
