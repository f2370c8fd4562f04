import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "salec-2d-public_b200"), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle library oracle/_ref/libsalec_ref.so is not built (needs the reference tree)")
    return ref


@pytest.fixture(scope="session")
def cuda_device():
    if not _has_cuda():
        pytest.fail("this test needs a CUDA device")
    return 0
