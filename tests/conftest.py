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
