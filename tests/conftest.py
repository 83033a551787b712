import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return torch.device("cuda")


@pytest.fixture(scope="session")
def ref():
    """The reference's own CUDA build (oracle/_ref), used as the bit-exact checker."""
    from oracle import build_ref
    m = build_ref.load("ref_rasterizer_C")
    if m is None:
        pytest.skip("reference build oracle/_ref/ref_rasterizer_C.so not present")
    return m
