import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def pk_table():
    from ezmock_b200.workloads import bbks_pk
    return bbks_pk()


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_16.npz"))


def has_ref():
    return all(os.path.exists(os.path.join(ROOT, "oracle", "_ref", f"libezref_f{p}.so"))
               for p in (32, 64))
