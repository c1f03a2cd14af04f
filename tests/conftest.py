import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / 'tests' / 'golden'


def pytest_configure(config):
    config.addinivalue_line(
        'markers', 'gpu: needs a CUDA GPU (sm_100a); run with -m gpu')


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason='no CUDA GPU in this process')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    return np.load(GOLDEN / f'{name}.npz')


@pytest.fixture(scope='session')
def golden_ab():
    return load_golden('ab')


@pytest.fixture(scope='session')
def golden_holo():
    return load_golden('holo')


@pytest.fixture(scope='session')
def golden_fit():
    return load_golden('fit')


@pytest.fixture(scope='session')
def golden_layered():
    return load_golden('layered')


@pytest.fixture(scope='session')
def golden_estimate():
    return load_golden('estimate')


@pytest.fixture(scope='session')
def golden_variants():
    return load_golden('variants')
