import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cx():
    """The C restatement oracle (oracle/cx_oracle.c)."""
    from oracle.oracle import CxOracle
    return CxOracle()


@pytest.fixture(scope="session")
def ref():
    """The reference operators compiled unmodified, if they were built."""
    from oracle.oracle import RefOracle
    if not RefOracle.available():
        pytest.skip("reference oracle (oracle/_ref) not built")
    return RefOracle()


@pytest.fixture(scope="session")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpetx_b200  # noqa: F401  (raises if the library is missing)
    return torch.device("cuda:0")
