import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def agal_lib():
    """The CUDA library, built in-tree when missing or stale."""
    from agal_b200 import build
    if not os.environ.get("AGAL_NO_BUILD"):
        try:
            build.build()
        except RuntimeError:
            # No nvcc on this machine: use the shipped library as is.
            pass
    from agal_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import orc
    orc.build()
    return orc.lib()
