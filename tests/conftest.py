import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def fgt():
    """The product library; GPU tests fail loudly when it is missing."""
    import fgt_b200
    if not os.path.exists(fgt_b200.LIB_PATH):
        from fgt_b200 import build as b
        b.build()
    fgt_b200.lib()
    return fgt_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def relerr(ref, approx):
    ref = np.asarray(ref).ravel()
    approx = np.asarray(approx).ravel()
    n = np.linalg.norm(ref)
    return float(np.linalg.norm(ref - approx) / (n if n > 0 else 1.0))
