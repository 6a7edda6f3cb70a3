import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "cosmo-nbody_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden_files():
    files = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    return [os.path.join(GOLDEN, f) for f in files]


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
