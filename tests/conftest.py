import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libchapsim_gpu.so")


@pytest.fixture(scope="session", autouse=True)
def _build_oracle():
    from oracle import pyoracle
    pyoracle.lib()
