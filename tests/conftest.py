import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def reference_file(rel: str):
    """A file of the reference checkout named by the FV_REFERENCE_DIR
    environment variable, or None when the variable is unset or the file is
    absent (tests that need it skip)."""
    base = os.environ.get("FV_REFERENCE_DIR")
    if not base:
        return None
    p = Path(base) / rel
    return p if p.exists() else None


sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfvb200.so")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def fv():
    from fvb200.build import build
    build()
    import fvb200
    return fvb200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
