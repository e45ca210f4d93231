"""pytest configuration: the `gpu` marker and shared helpers."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libfdzb.so")


@pytest.fixture(scope="session")
def fdzb():
    return importlib.import_module("4dzb_b200")


@pytest.fixture(scope="session")
def scenes():
    return importlib.import_module("4dzb_b200.scenes")


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return True
