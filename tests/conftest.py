import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def small_phantom():
    from cs_dmri_b200.phantom import make_phantom
    return make_phantom((8, 8, 4), seed=7)


@pytest.fixture(scope="session")
def lib_built():
    from cs_dmri_b200.build import build
    build()
    return True
