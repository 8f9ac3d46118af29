"""pytest configuration: the `gpu` marker and session-wide native builds."""
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import helpers  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def native():
    """Builds libzindex_b200.so, the tools and the oracle (incremental)."""
    helpers.build_native()
    return True


@pytest.fixture(scope="session")
def oracle(native):
    return helpers.Oracle()


def _cuda_ok() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(native):
    if not _cuda_ok():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return 0
