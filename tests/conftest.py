import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the sm_100a path")


@pytest.fixture(scope="session")
def lib():
    """libsundog.so, compiled in-tree when missing (never a CPU fallback)."""
    from sundog_b200 import abi, build
    if not os.path.isfile(abi.LIB_PATH):
        build.build()
    return abi.load()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    if not os.path.isfile(oracle.LIB_PATH):
        oracle.build()
    return oracle.load()


@pytest.fixture(scope="session")
def asset_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("assets"))

