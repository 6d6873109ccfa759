import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import tcref
    if not tcref.available():
        pytest.skip("reference library oracle/_ref/libtcref.so not built")
    return tcref.ref_lib()
