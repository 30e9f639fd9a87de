import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def load_package():
    import stwo_gpu_b200
    return stwo_gpu_b200


sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libstwo_b200.so")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O  # noqa: E402  (oracle/oracle.py, test infrastructure)
    O.lib()
    return O


@pytest.fixture(scope="session")
def stwo():
    return load_package()
