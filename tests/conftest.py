import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _have_cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_CUDA = _have_cuda()


@pytest.fixture(scope="session")
def ndlib():
    """The in-tree CUDA library (loaded, never built, on a GPU machine)."""
    from numericdream_b200 import runtime, build

    if not os.path.exists(runtime.LIB_PATH) and not HAVE_CUDA:
        build.build()
    return runtime.load_library()


@pytest.fixture(scope="session")
def ctx(ndlib):
    if not HAVE_CUDA:
        pytest.skip("no CUDA device")
    from numericdream_b200 import runtime

    c = runtime.Context(0)
    yield c
    c.close()
