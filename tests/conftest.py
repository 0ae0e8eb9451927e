import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def small_case():
    """6x4-element mesh of the small half-space layout (strip 2) and two (f, py) pairs."""
    from fem25_b200 import synth
    mesh, pairs, _ = synth.make_config(0, nx=8, nz=5)
    return mesh, pairs
