import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("cfpq-on-gpgpu_b200")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o  # the checker (CPU restatement)

    o.lib()
    return o


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.capi.Context(0)
    yield c
    c.close()
