import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def port_lib():
    from oracle import oracle
    return oracle.port()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import oracle
    lib = oracle.reference()
    if lib is None:
        pytest.skip("reference build oracle/_ref/librhref.so not present")
    return lib


@pytest.fixture(scope="session")
def ref_gc_lib():
    from oracle import oracle
    lib = oracle.reference_gc()
    if lib is None:
        pytest.skip("reference build oracle/_ref/librhref_gc.so not present")
    return lib
