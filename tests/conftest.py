import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests against the oracle")


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference_kernels():
    from oracle.oracle import Reference
    if not Reference.available():
        import oracle.oracle as o
        o.build()
    if not Reference.available():
        pytest.skip("reference kernels not built (pTatin3d sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ptatin3d_b200 import lib
    lib()  # raises if libp3d_b200.so is missing: no CPU fallback
    return torch.device("cuda", 0)
