import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def engine_lib():
    import __graft_entry__ as ge
    ge.build_engine()
    from ermod_openacc_b200 import _capi
    return _capi.load_library()


@pytest.fixture(scope="session")
def slvfe_oracle():
    import slvfe_oracle
    return slvfe_oracle
