import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: full-size workload")


@pytest.fixture(scope="session")
def ctx():
    import distance_transform_benchmarks_b200 as dtb
    c = dtb.Context(0)
    yield c
    c.close()
