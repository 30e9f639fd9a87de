import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "stwo-gpu_b200")


def load_package():
    """Import the package directory stwo-gpu_b200/ as module `stwo_gpu_b200`."""
    if "stwo_gpu_b200" in sys.modules:
        return sys.modules["stwo_gpu_b200"]
    spec = importlib.util.spec_from_file_location(
        "stwo_gpu_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["stwo_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


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
