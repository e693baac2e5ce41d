import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a)')


def package():
    """The product package (its directory name is not a Python identifier, so import it by name)."""
    return importlib.import_module('hahenn-_b200')


@pytest.fixture(scope='session')
def pkg():
    return package()
