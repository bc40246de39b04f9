import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def rel_l2(a, b) -> float:
    """Relative L2 error ||a - b|| / ||b|| (0 when both vanish)."""
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    na = np.linalg.norm((a - b).ravel())
    r = float(na) if nb == 0 else float(na / nb)
    # a NaN would slip through max()-style accumulation; report it as infinite
    return r if np.isfinite(r) else float("inf")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def sns():
    import spectral_upcxx_b200 as S
    S.lib()
    return S


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device; run it with -m gpu on a GPU host")
    return torch.device("cuda", 0)
