import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and libptbgpu.so (parity tests through the C-ABI)")


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests (fails loudly without the library)."""
    from ptb_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def water8():
    from ptb_b200 import synth
    return synth.water_cluster(8, seed=5)


@pytest.fixture(scope="session")
def water32():
    from ptb_b200 import synth
    return synth.water_cluster(32, seed=1)
