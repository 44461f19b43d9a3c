import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import RefLib, ref_available
    if not ref_available():
        pytest.skip("reference CPU library not built")
    return RefLib()


@pytest.fixture(scope="session")
def ctx():
    from structure_b200 import Context
    return Context(0)
