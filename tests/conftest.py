import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: larger sizes")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not cuda_available():
        pytest.fail("this test needs a CUDA device; run it with -m gpu on a GPU host")
    import torch

    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def ref_dir():
    """oracle/_ref (the reference built from its sources), or skip when absent."""
    d = REPO / "oracle" / "_ref"
    if not any(d.glob("pycusaxs_cuda*.so")):
        pytest.skip("reference build oracle/_ref not present")
    return d
