import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "pytorch-tcuscan_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200, sm_100a) device")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return np.load(os.path.join(REPO, "tests", "golden", "golden.npz"))


def _ensure_lib():
    """Build libtcuscan.so in-tree when it is missing or older than its sources
    (nvcc cross-compiles on CPU; incremental).  On a machine without nvcc the
    prebuilt library is used as is."""
    lib = os.path.join(PKG, "lib", "libtcuscan.so")
    sys.path.insert(0, PKG)
    import build as _b

    if not os.path.exists(lib) or os.path.exists(_b.NVCC):
        _b.build()
    return lib


LIB_PATH = _ensure_lib()


def cuda_ok():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
