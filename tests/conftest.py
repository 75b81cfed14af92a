"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the C-ABI library")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ygmod():
    from yandasoft_b200 import build, gridder
    build.build()
    gridder.load()
    return gridder


@pytest.fixture(scope="session")
def c0_small():
    """Config-0 layout, shortened to 10 minutes (37,800 rows x 8 channels)."""
    from yandasoft_b200 import simulate
    ds, p = simulate.config0(duration_s=600.0)
    return ds, p
