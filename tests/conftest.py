import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden128():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "c128_fixtures.npz")))


@pytest.fixture(scope="session")
def golden64():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "c64_fixtures.npz")))
