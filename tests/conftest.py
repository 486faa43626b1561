"""Shared pytest setup: the `gpu` marker and a library session fixture."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 GPU (runs the CUDA sm_100a library)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return np.load(os.path.join(ROOT, "tests", "golden", "evsl_ref_golden.npz"))


@pytest.fixture(scope="session")
def gpu_lib():
    """One EVSLStart session shared by the GPU tests (fails loudly without a GPU)."""
    import evsl_b200

    lib = evsl_b200.Library()
    yield lib
    lib.finish()
