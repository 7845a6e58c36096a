"""Test configuration: the `gpu` marker and the one-time in-tree builds.

CPU tests (-m "not gpu") check the oracle against GALIC's own C and the
committed golden fixtures, the host-side logic, and that libgalic_cuda.so
loads and exports every symbol of include/galic_gpu.h.  GPU tests (-m gpu)
call the CUDA path through the C ABI and compare it with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    from galic_b200 import build
    import oracle_lib

    build.build()
    oracle_lib.build_oracle()
    yield


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
