import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def train_stats(oracle):
    """Stats of the homogeneous 128x128 training area (R=1, coherence 0.6),
    patches {3,5,7}, scales {1,3}, built by the oracle."""
    from despeckcl_b200 import synthetic

    a1, a2, ph = synthetic.training_area(128, seed=7)
    return oracle.training_insar(a1, a2, ph, [3, 5, 7], [1, 3])
