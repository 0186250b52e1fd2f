import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = 'hybridpendulum-up_b200'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


def load_pkg():
    """Import the product package (its directory name has a hyphen)."""
    return importlib.import_module(PKG_NAME)


@pytest.fixture(scope='session')
def hp():
    return load_pkg()
