import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build()
    return Oracle()


@pytest.fixture(scope="session")
def refcpu(oracle):
    from oracle.oracle import RefCPU
    try:
        return RefCPU()
    except FileNotFoundError:
        pytest.skip("reference QSR.cpp build (oracle/_ref) not available")


@pytest.fixture(scope="session")
def lib():
    from lcdrsimulator_b200.build import build
    build()
    import lcdrsimulator_b200 as L
    return L.load_library()
