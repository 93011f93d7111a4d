import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def ctx():
    """One libnsat context on cuda:0 for the GPU tests (fails loudly without a device)."""
    from naivesat_b200 import api
    c = api.Context(0)
    yield c
    c.close()


# test modules import helpers from one another (e.g. test_gpu_shard uses
# test_shard.oracle_sub)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)
