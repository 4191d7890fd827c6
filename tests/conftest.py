import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")
    config.addinivalue_line("markers", "slow: long-running solve")


def have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def rq():
    import rans_uq_b200

    rans_uq_b200.lib()  # the CUDA library must load: there is no fallback
    return rans_uq_b200


@pytest.fixture(scope="session")
def checker():
    from oracle import checker as ck

    if not ck.have("oracle"):
        pytest.skip("oracle/librq_oracle.so not built (make -C oracle)")
    return ck
