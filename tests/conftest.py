import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, 'oracle')):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (run with -m gpu)')


@pytest.fixture(scope='session')
def av1b():
    import av1ongpu_b200
    return av1ongpu_b200


@pytest.fixture(scope='session')
def oracle():
    import refdec
    if not refdec.available():
        pytest.skip('oracle/_ref/libav1ref.so is not built (make -C oracle)')
    return refdec
