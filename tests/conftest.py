import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def lbm():
    import lbm_ddf_b200

    lbm_ddf_b200.lib()
    return lbm_ddf_b200
