import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a B200 GPU (runs the CUDA engine through the C-ABI)')


def golden(name):
    with np.load(os.path.join(HERE, 'golden', name + '.npz'), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope='session')
def ora():
    from oracle_lib import Oracle
    return Oracle()


@pytest.fixture(scope='session')
def ctx():
    """GPU context through the C-ABI; fails (does not skip) if the engine
    cannot load or no GPU answers, so a silent CPU fallback cannot pass."""
    from hfpx3d_b200 import build, engine
    build.build()
    c = engine.Context(0)
    yield c
    c.close()
