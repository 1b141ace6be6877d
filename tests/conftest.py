import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through libcuda_replace.so")


@pytest.fixture(scope="session")
def cr_lib():
    """The CUDA library, built in-tree. GPU tests fail loudly when it cannot be loaded."""
    from cuda_replace_b200 import build as B
    from cuda_replace_b200.cuda_replace_wrapper import CudaReplaceLib
    if not B.LIB_PATH.exists():
        B.build()
    return CudaReplaceLib(str(B.LIB_PATH))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build_oracle()
    return O


@pytest.fixture(scope="session")
def fake_lib_path():
    """A CPU implementation of the C ABI built from the C oracle (test double only)."""
    from tests import fake_capi
    return fake_capi.build()
