import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "zinc-plus_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def zipgpu():
    import zipgpu

    zipgpu.lib()
    return zipgpu


@pytest.fixture(scope="session")
def ctx(zipgpu):
    c = zipgpu.Context(0)
    yield c
    c.close()


@pytest.fixture
def rng():
    return np.random.default_rng(0x5A1F)
