import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libabcmb_b200.so")


@pytest.fixture(scope="session")
def c1_small():
    """C1 cosmology with 40 k modes: seconds on the oracle."""
    from abcmb_b200 import configs
    return configs.c1(nk=40, xe_layout="compact").build()


@pytest.fixture(scope="session")
def c1_oracle(c1_small):
    from oracle import oracle
    rc, pt, ks = oracle.pert_forward(c1_small.batch, c1_small.pert_settings())
    assert rc == 0
    return pt, ks
