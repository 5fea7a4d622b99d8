import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


def ref_lib(edge):
    """ARGOT's own C (O1) for an edge^3 mesh, or skip when neither the
    prebuilt library nor the reference sources are present."""
    from oracle import build
    from oracle.oracle import RefLib
    if not os.path.exists(build.ref_lib_path(edge)) and not build.reference_available():
        pytest.skip("reference build unavailable")
    return RefLib(edge)


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
