import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hybrid-final_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    lib = os.path.join(PKG, "lib", "libhpic.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    olib = os.path.join(REPO, "oracle", "_build", "liboracle.so")
    if not os.path.exists(olib):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")
