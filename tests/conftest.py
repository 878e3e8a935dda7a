"""Shared test set-up.  Tests that need a B200 carry @pytest.mark.gpu."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc
    orc.load_oracle()
    return orc


@pytest.fixture(scope="session")
def mdwt_lib():
    from mdwtracker_b200 import load_library
    return load_library()
