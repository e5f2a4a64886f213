import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def V():
    import vortexlab_b200
    return vortexlab_b200


@pytest.fixture(scope="session")
def O():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu(V):
    if V.device_count() == 0:
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return V


@pytest.fixture(scope="session")
def published():
    """The reference's published known answers (tests/golden/published.json, made by
    tests/golden/make_published.py from docs/report/index.html:59 and README.md:182-188)."""
    with open(os.path.join(TESTS, "golden", "published.json")) as f:
        return json.load(f)
