import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.build import build_oracle

    build_oracle()
    from oracle import oracle as O

    O.load()
    return O


@pytest.fixture(scope="session")
def cuda_lib():
    """The built CUDA library on a GPU machine (GPU tests only)."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    from slosh_b200.build import build_library, up_to_date

    if not up_to_date():
        build_library()
    from slosh_b200 import _lib

    return _lib.load()
