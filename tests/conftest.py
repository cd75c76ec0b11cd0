import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def _cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def built():
    """Build the CUDA library and the CPU oracle if stale (no GPU needed)."""
    from kh_simulations_b200 import build

    import oracle

    build.build()
    if not oracle.ORACLE_LIB.exists():
        oracle.build(ref=False)
    return True


@pytest.fixture(scope="session")
def cuda(built):
    if not _cuda():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session")
def orc(built):
    from oracle import Oracle

    return Oracle()
