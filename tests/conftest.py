import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden_host():
    import numpy as np
    return np.load(os.path.join(GOLDEN, "ref_host.npz"))


@pytest.fixture(scope="session")
def golden_abi():
    import numpy as np
    return np.load(os.path.join(GOLDEN, "ref_gpu_abi.npz"))
