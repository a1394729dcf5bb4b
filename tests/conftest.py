import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: large full-size cases")


@pytest.fixture(scope="session")
def ctx():
    from hpcsharp_b200 import build, native

    build.build_all()
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle
