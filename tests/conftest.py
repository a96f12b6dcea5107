import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "lbmengine.jl_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liblbm_b200.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def lib():
    """liblbm_b200.so (built in-tree if missing; loading never falls back to CPU)."""
    import importlib.util
    from lbmengine import _capi
    spec = importlib.util.spec_from_file_location("lbm_b200_build", os.path.join(PKG, "build.py"))
    libbuild = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(libbuild)
    libbuild.build()
    return _capi.load()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    oracle.load()
    return oracle
