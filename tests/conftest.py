import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def oracle():
    from ftoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from ftoracle import REF_DRIVER_SO, Reference
    if not os.path.exists(REF_DRIVER_SO):
        pytest.skip("reference build absent (make -C oracle ref)")
    return Reference()


@pytest.fixture(scope="session")
def device():
    import fainttrail_b200 as ftb
    return ftb.Device()


@pytest.fixture(scope="session")
def backend(device):
    import fainttrail_b200 as ftb
    return ftb.make_backend("b200", device)


def golden(name):
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", name), allow_pickle=False)
