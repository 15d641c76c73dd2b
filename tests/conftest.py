import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the sm_100a kernels")


@pytest.fixture(scope="session")
def dumps(tmp_path_factory):
    """Synthetic iharm dumps, generated once per session from their seeds."""
    from tests import common
    d = tmp_path_factory.mktemp("dumps")
    return common.DumpCache(str(d))
