"""pytest set-up: the `gpu` marker (tests that need a B200) and import paths for the package and the oracle."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200); run with -m gpu")


@pytest.fixture(scope="session")
def ws():
    import weavesim_b200
    return weavesim_b200


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle

