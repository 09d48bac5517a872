import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dg-mpi_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_built():
    if not os.path.exists(os.path.join(ORACLE, "_build", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    if not os.path.exists(os.path.join(PKG, "_build", "libdg_b200.so")):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)


_ensure_built()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as f:
        return json.load(f)
