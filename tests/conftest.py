import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def native_lib():
    from segmentctscans_b200.build import build_native

    build_native()
    from segmentctscans_b200 import _native

    return _native.host_lib()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle.build import build_oracle

    build_oracle()
    from oracle import oracle

    return oracle


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
