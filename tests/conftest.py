import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session")
def gpu_lib(cuda_ok):
    from sdot_b200 import build

    build.build()
    from sdot_b200 import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import ref

    ref.build()
    if not ref.available():
        pytest.skip("compiled reference oracle not available")
    return ref
