import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def engine_lib():
    from mpdpft_b200 import engine
    return engine.load()


@pytest.fixture(scope="session")
def eng():
    """The engine module with its CUDA library loaded."""
    from mpdpft_b200 import engine
    engine.load()
    return engine
