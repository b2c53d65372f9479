import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ref():
    """The reference itself (its Fortran translated to C, oracle/ref.py)."""
    from oracle import ref as R
    R.build()
    if not R.available():
        pytest.fail("oracle/_ref/libfmm2d_ref.so missing: run `make -C oracle ref` where the "
                    "reference's sources are")
    return R


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import fmm2d_b200
    fmm2d_b200._lib.lib()  # loud failure if the library is missing
    return torch.device("cuda:0")


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
