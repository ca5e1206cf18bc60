import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a)')


GOLDEN = ROOT / 'tests' / 'golden'


@pytest.fixture(scope='session')
def golden():
    return GOLDEN
