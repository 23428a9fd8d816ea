import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def native_built():
    from co_cultivation_metabolic_atlas_b200 import build
    build.build()
    return build.LIB


@pytest.fixture
def forbid_cpu_optimizers(monkeypatch):
    import scipy.optimize

    def forbidden(*_a, **_k):
        raise AssertionError("CPU optimizer was called")
    monkeypatch.setattr(scipy.optimize, "linprog", forbidden)
