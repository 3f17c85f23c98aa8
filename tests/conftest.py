import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


_HAS_GPU = None


def has_gpu():
    global _HAS_GPU
    if _HAS_GPU is None:
        try:
            import torch
            _HAS_GPU = bool(torch.cuda.is_available())
        except Exception:
            _HAS_GPU = False
    return _HAS_GPU


@pytest.fixture(scope="session")
def gpu_lib():
    """The built C-ABI library.  Missing library = failure, not a skip."""
    if not has_gpu():
        pytest.skip("no CUDA device in this process")
    from multiphaselb_b200 import build, load_library
    build.build()
    return load_library()
