import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_checkers():
    """Build the CPU restatement (and the reference, where its sources are
    present) once per session; the GPU library is built by __graft_entry__."""
    from oracle import pyref

    if not pyref.oracle_available():
        pyref.build(ref=True)
    yield


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
