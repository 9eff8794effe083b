import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size configuration (runs in tens of seconds)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def libisf_path():
    import __graft_entry__ as ge
    return ge.load_builder().build()


@pytest.fixture(scope="session")
def isfpkg(libisf_path):
    import __graft_entry__ as ge
    return ge.load_package()


@pytest.fixture(scope="session")
def cfgs(isfpkg):
    import importlib
    return importlib.import_module(isfpkg.__name__ + ".configs")
