import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than ~30 s")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built():
    """Native libraries, built in-tree if missing (nvcc cross-compiles without a GPU)."""
    from igap4standard_b200 import build
    build.build()
    return True


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle library oracle/_ref/libref_iga.so not built")
    return ref
