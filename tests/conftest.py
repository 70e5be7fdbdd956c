import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# Reference unit constants (pScientific/__extensions__/cinclude/Units.h:27,37 and Constants.h:15).
ANGSTROM_TO_BOHR = 1.0e-10 / 5.291772083e-11
HARTREE_TO_KJMOL = 2625.5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_device():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return 0
