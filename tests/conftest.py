import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import pm_oracle
    pm_oracle.lib()
    return pm_oracle


@pytest.fixture(scope="session")
def pm():
    """The engine; GPU tests fail (not skip) if it is missing on a GPU box."""
    import polymer_b200
    if not have_gpu():
        pytest.skip("no CUDA device")
    polymer_b200.lib()
    return polymer_b200
