import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); the parity tests proper")
    config.addinivalue_line("markers", "slow: longer CPU-oracle runs")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """The C restatement always builds (gcc only); the reference oracle only
    where the reference sources are checked out."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    yield
