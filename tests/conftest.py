"""pytest configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs the oracle against the golden fixtures, the host pattern build
through the C ABI and the host logic; ``-m gpu`` runs the parity tests of the CUDA path
against the oracle (they need a B200 and the built library).
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhippymfem_b200.so")


def golden_cases():
    return sorted(f for f in os.listdir(GOLDEN) if f.startswith("pattern_") and f.endswith(".npz"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
