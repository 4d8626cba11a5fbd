import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def hd(torch_cuda):
    import hygondoubleblockedfactorizations_b200 as hd
    hd.lib()  # fails loudly when the CUDA library is missing
    return hd


@pytest.fixture()
def handle(hd, torch_cuda):
    h = hd.Handle(torch_cuda.cuda.current_stream().cuda_stream)
    yield h
    torch_cuda.cuda.synchronize()
    h.close()
