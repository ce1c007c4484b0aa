import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


@pytest.fixture(scope="session")
def gpu_ctx():
    """One device context for the GPU tests. Fails (does not skip) when no
    device is present: a GPU test that silently skipped would hide a missing
    native path."""
    from calamarijoins_b200 import Context
    ctx = Context()
    yield ctx
    ctx.close()
