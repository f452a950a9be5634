import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("workloads"))


@pytest.fixture(scope="session", autouse=True)
def built():
    from cgbdsm_b200 import build as b
    b.build()
    from oracle import bind
    bind.build(ref=True)
    return True
