import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tblite-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PARAMS = os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco.tbp")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def params_path():
    return PARAMS


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.Oracle(PARAMS)


@pytest.fixture(scope="session")
def gpu_calc():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tblite_b200 import Calculator
    return Calculator(PARAMS)
