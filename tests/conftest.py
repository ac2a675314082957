import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def small_channel():
    from myfvcomcode_b200 import cases
    return cases.estuary_channel(nx=24, ny=6, kb=6, lx=4800.0, ly=1200.0, IRAMP=10)


@pytest.fixture(scope="session")
def small_channel_edge():
    from myfvcomcode_b200 import cases
    return cases.estuary_channel(nx=24, ny=6, kb=6, lx=4800.0, ly=1200.0, IRAMP=10,
                                 river_location="edge")


@pytest.fixture(scope="session")
def small_coastal():
    from myfvcomcode_b200 import cases
    return cases.coastal_mesh(npts=1500, kb=7, lx=20000.0, ly=10000.0, seed=7, IRAMP=20)
