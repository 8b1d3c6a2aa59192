import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")
    config.addinivalue_line("markers", "slow: long statistical run")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden16():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "golden_w16.npz")))


@pytest.fixture(scope="session")
def golden8():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "golden_w8.npz")))


@pytest.fixture(scope="session")
def c3_fixtures():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "c3_sha.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def gpu():
    """The native library with at least one CUDA device; GPU tests fail loudly without them."""
    import computational_physics_b200 as cp
    n = cp.device_count()
    if n < 1:
        pytest.fail("no CUDA device visible to libswb200.so")
    return cp
