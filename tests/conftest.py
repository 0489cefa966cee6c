"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built engine."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, 'tests', 'golden', 'golden.npz')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built engine')


@pytest.fixture(scope='session')
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope='session')
def skeletal():
    from multifil_jax_b200 import get_skeletal_params
    return get_skeletal_params()


@pytest.fixture(scope='session')
def engine():
    from multifil_jax_b200.engine import get_engine
    return get_engine(0)
