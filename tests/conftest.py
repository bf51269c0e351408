import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built CUDA library")


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


# integer-weighted cases: every FP64 sum is exact, so results are bit-exact
INTEGER_CASES = {"planted_int", "rmat_unit", "rmat_int", "sparse_isolated", "selfloop_int"}


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def nido_lib():
    from nido_b200 import capi
    capi.lib()
    return capi


@pytest.fixture(scope="session")
def ctx(nido_lib):
    c = nido_lib.Context(0)
    yield c
    c.close()
