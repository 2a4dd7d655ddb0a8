import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _checkers_built():
    """Compile the oracle restatement (and the reference core when its sources
    are present) once per session."""
    from oracle import driver
    if not driver.available("oracle") or (os.path.isdir(driver.REF_SRC) and not driver.available("ref")):
        driver.build(ref=True)
    yield


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
