# -*- coding: utf-8 -*-
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, 'dgfs-be-solver_b200')):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')
SPHDESIGN = os.path.join(ROOT, 'dgfs-be-solver_b200', 'frfs_b200', 'data',
                         'sphericaldesign')


def pytest_configure(config):
    config.addinivalue_line(
        'markers', 'gpu: needs a B200 (runs the CUDA library)')


@pytest.fixture(scope='session')
def golden_dir():
    return GOLDEN
