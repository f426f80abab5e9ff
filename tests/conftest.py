import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port():
    from oracle.checkers import Port

    return Port()


@pytest.fixture(scope="session")
def reference():
    from oracle.checkers import Reference

    if not Reference.available():
        pytest.skip("the reference painter library (oracle/_ref) is not built here")
    return Reference()


@pytest.fixture(scope="session")
def require_gpu():
    if not cuda_available():
        pytest.fail("a CUDA device is required for tests marked gpu")
    os.environ.setdefault("NTRACE_NO_BUILD", "1")
