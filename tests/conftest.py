import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")
os.environ.setdefault("MZB_QUIET", "1")

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import loader
    return loader.load_kernels()


@pytest.fixture(scope="session")
def oracle_path():
    from oracle import loader
    return loader.oracle_path()


@pytest.fixture(scope="session")
def product_path():
    """Path of the built product library (built here if missing; never a fallback)."""
    from maze_poisson_b200 import build, library_path
    path = library_path()
    if not os.path.exists(path):
        build.build()
    return path
