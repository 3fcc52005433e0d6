import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

ufc = __graft_entry__.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (parity tests through the C-ABI)")


@pytest.fixture(scope="session")
def pkg():
    return ufc


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    return O
