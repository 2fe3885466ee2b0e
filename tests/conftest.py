import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200")
ORACLE = os.path.join(ROOT, "oracle")
TESTS = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(TESTS, "golden")
for p in (PKG, ORACLE, TESTS, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_built():
    import build_oracle as oracle_build
    return oracle_build.build()


@pytest.fixture(scope="session")
def cgfd_lib():
    """The CUDA product library; fails loudly (no CPU fallback)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("cgfd_pkg_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    import cgfd
    return cgfd.load_library()
