import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import pyoracle
    pyoracle.load()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The in-tree CUDA library; a GPU test fails loudly if it is missing."""
    from fortran_loadfile_mitiwing_b200 import _abi, build
    build.build()
    return _abi.load_library()
