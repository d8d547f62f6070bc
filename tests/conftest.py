import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "ref: needs the reference build under oracle/_ref")


@pytest.fixture(scope="session")
def ref():
    from oracle import ref as _ref
    if not _ref.available():
        pytest.skip("reference oracle (oracle/_ref/libccnn_ref.so) not built")
    return _ref
