import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_vectors.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libnan_b200.so")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def device():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import nan_b200

    return nan_b200.Device(0)
