import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def tmp_root(tmp_path_factory):
    base = "/dev/shm" if os.path.isdir("/dev/shm") and os.access("/dev/shm", os.W_OK) else None
    if base:
        import tempfile
        d = tempfile.mkdtemp(prefix="egtb_test_", dir=base)
        yield d
        import shutil
        shutil.rmtree(d, ignore_errors=True)
    else:
        yield str(tmp_path_factory.mktemp("egtb"))


@pytest.fixture(scope="module", autouse=True)
def _release_device_memory_after_module():
    """The library keeps its build buffers (arena, sets, indexes, books) at
    the size of the largest table built; after each test module they are
    freed (egtb_release), so a module that built a large table leaves the
    device's memory to the next one."""
    yield
    import importlib
    N = importlib.import_module("2048endgametablebase_b200._native")
    if N._lib is None:
        return
    try:
        import torch
        if not torch.cuda.is_available():
            return
        for d in range(torch.cuda.device_count()):
            N.release(d)
        torch.cuda.empty_cache()
    except Exception:  # noqa: BLE001 - a module whose device work failed reports that itself
        pass
