import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")
    config.addinivalue_line("markers", "reference: needs the reference-core checker library (oracle/_ref)")


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def reference_available():
    from oracle import REF_LIB

    if not REF_LIB.is_file():
        pytest.skip("reference-core checker library not built")
    return True
