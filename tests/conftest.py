import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the B200 kernels)")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """The oracle libraries are test infrastructure; build them if missing (CPU only)."""
    for sub, lib in (("oracle", "liboracle.so"), ("workloads", "libvxgen.so")):
        if not os.path.exists(os.path.join(ROOT, sub, lib)):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, sub)], check=True)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
