import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "golden.npz")
    return dict(np.load(path, allow_pickle=False))


@pytest.fixture(scope="session")
def golden_models():
    """The reference's CTDS variants (CpuSatTanh, bias term) on golden.npz's problems."""
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "golden_models.npz")
    return dict(np.load(path, allow_pickle=False))
