import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfwt.so")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def fwt():
    import fastweavturb_b200 as F

    F.library()
    return F
