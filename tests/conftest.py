import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _built() -> bool:
    return os.path.exists(os.path.join(ROOT, "hotspot_b200", "libhotspot_b200.so")) and \
        os.path.exists(os.path.join(ROOT, "oracle", "_build", "libgrid_oracle.so"))


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """Build the product library and the oracle once if they are missing."""
    if not _built():
        import __graft_entry__
        __graft_entry__.build()
    yield


@pytest.fixture
def workdir(tmp_path):
    return str(tmp_path)


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
