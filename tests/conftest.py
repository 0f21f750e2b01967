import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def ref():
    from oracle.bindings import RefLib, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built (the reference checkout is needed to build it)")
    return RefLib()


@pytest.fixture(scope="session")
def orc():
    from oracle.bindings import OracleLib, oracle_available

    if not oracle_available():
        pytest.skip("oracle/liboracle.so not built (make -C oracle)")
    return OracleLib()
