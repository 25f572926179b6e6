import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _ensure_built():
    """Builds the native libraries and the oracle when they are missing (the
    GPU run uses the prebuilt files that travel with the repository)."""
    from spmv_b200 import build as B
    import oracle
    if not B.LIB.exists() or not B.GEN.exists():
        B.build()
    if not oracle.LIB_PATH.exists():
        oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return 0
