import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("match-series_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    import msor
    msor.lib()
    return msor


@pytest.fixture(scope="session")
def gpu():
    import msgpu
    from msgpu import build
    build.build()
    ctx = msgpu.Context(0)
    yield ctx
    ctx.close()


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name))
