import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (built on demand from oracle/accel_oracle.c)."""
    from oracle import pyoracle
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return pyoracle


@pytest.fixture(scope="session")
def ablib():
    from presto_b200 import build
    build.build()
    import presto_b200
    return presto_b200


@pytest.fixture(scope="session")
def ctx(ablib):
    c = ablib.Context(0)
    yield c
    c.close()
