"""Test configuration: the `gpu` marker (tests that need a CUDA device, run on a B200) and the paths."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (sm_100a); run with -m gpu on a B200')


@pytest.fixture(scope='session')
def root():
    return ROOT
