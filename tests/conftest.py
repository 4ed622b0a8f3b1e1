import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def mflib():
    """The product library, built in-tree if missing (nvcc cross-compiles without a GPU)."""
    from markerfree_b200 import build
    build.build()
    import markerfree_b200 as mf
    mf.lib()
    return mf


@pytest.fixture(scope="session")
def ctx(mflib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    c = mflib.Context(0)
    yield c
    c.close()
