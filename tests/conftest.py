import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
# The reference's source tree, read only by CPU tests that load its pure-Python
# modules or stub files; they skip when it is absent (as on a GPU box).  It is
# PROPAQ_REFERENCE, else a directory named `reference` beside the repository.
REFERENCE_TREE = Path(os.environ.get("PROPAQ_REFERENCE") or ROOT.parent / "reference")
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle_client import Oracle

    return Oracle.load()


@pytest.fixture(scope="session")
def gpu_engine():
    if not _cuda_available():
        pytest.skip("no CUDA device")
    from propaq_b200 import _native

    return _native.engine(0)
