import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")
    config.addinivalue_line("markers", "slow: long CPU reference runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle.refio import ORACLE_SO, Oracle

    if not os.path.exists(ORACLE_SO):
        pytest.skip("oracle/liboracle.so not built")
    return Oracle()


@pytest.fixture(scope="session")
def gpu_ctx():
    from whirplonk_b200 import Context

    ctx = Context(0)
    yield ctx
    ctx.close()
