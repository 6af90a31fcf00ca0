import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def water2():
    return golden("ref_water2.npz")


@pytest.fixture(scope="session")
def chain12():
    return golden("ref_chain12.npz")


def shell_table(fx):
    from proteindf_b200 import basis
    return basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"], basis.load_basis("cc-pVDZ"))
