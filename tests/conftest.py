import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build(reference=False)
    return O


def golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
