import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "flash-x_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import fx_oracle
    fx_oracle.lib()
    return fx_oracle


@pytest.fixture(scope="session")
def need_gpu():
    if not has_gpu():
        pytest.fail("GPU test run without a visible CUDA device")
