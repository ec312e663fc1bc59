import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle_lib():
    from tests.util import load_oracle
    return load_oracle()


@pytest.fixture(scope="session")
def ref_lib():
    from tests.util import load_ref
    lib = load_ref()
    if lib is None:
        pytest.skip("compiled reference (oracle/_ref) not present")
    return lib


@pytest.fixture(scope="session")
def gpu_lib():
    from tests.util import load_product
    return load_product()
