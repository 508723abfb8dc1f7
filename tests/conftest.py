"""Shared test setup: the `gpu` marker, and the built native libraries."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) CUDA device")


def _ensure_built():
    from natray_b200 import build as nb
    from oracle import build as ob
    nb.build()
    ob.build()


_ensure_built()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_threads():
    from oracle.py import set_threads
    set_threads(int(os.environ.get("NTR_ORACLE_THREADS", "0")))
    return True
