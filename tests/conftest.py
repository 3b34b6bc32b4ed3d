"""Test configuration: the `gpu` marker and build fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's golden
outputs, the host logic of the library and its exported C ABI.  GPU tests
(-m gpu) compare the CUDA paths with the oracle through the C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def mq():
    from mqct_b200 import build
    build.build()
    import mqct_b200
    return mqct_b200


@pytest.fixture(scope="session")
def gpu_available(mq):
    from mqct_b200 import _abi
    if _abi.lib().mqct_device_count() <= 0:
        pytest.fail("GPU test selected but no CUDA device is visible")
    return True
