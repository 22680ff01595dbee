"""pytest configuration: the `gpu` mark (tests that need a CUDA device and the built library) and the paths the
tests use. Tests without the mark run on the CPU alone (`pytest -m "not gpu"`)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
for p in (ROOT, os.path.join(ROOT, 'oracle')):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a) and the built fastsar_b200 library')
    config.addinivalue_line('markers', 'slow: a longer CPU test')


@pytest.fixture(scope='session')
def golden():
    """Loader of a golden fixture by name: golden('plan_small2') -> the npz's dict."""
    import numpy as np
    cache = {}

    def load(name):
        if name not in cache:
            with np.load(os.path.join(GOLDEN, name + '.npz')) as z:
                cache[name] = {k: z[k] for k in z.files}
        return cache[name]
    return load


@pytest.fixture(scope='session')
def oracle_lib():
    """The oracle module with its C library built (make -C oracle)."""
    import subprocess
    import oracle as O
    if not O.available('port'):
        subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)
    return O
