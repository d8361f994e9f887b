import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "filianore-core_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ref_tables():
    return dict(np.load(os.path.join(GOLDEN, "spectral_tables.npz")))


@pytest.fixture(scope="session")
def orc_tables(ref_tables):
    import oracle
    return oracle.Tables(ref_tables)
