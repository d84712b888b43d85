import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdftk.so")
    config.addinivalue_line("markers", "slow: long-running parity case")


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not generated")
    return dict(np.load(path, allow_pickle=False))


@pytest.fixture(scope="session")
def golden_h2o():
    return load_golden("h2o.npz")


@pytest.fixture(scope="session")
def golden_c10h22():
    return load_golden("c10h22.npz")


@pytest.fixture(scope="session")
def golden_h2o64():
    return load_golden("h2o64_sample.npz")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.lib()
    return oracle
