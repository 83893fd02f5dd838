import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "pristine.npz"))


def golden_csr(golden, stem):
    import scipy.sparse as sp
    sh = golden[stem + "__shape"]
    return sp.csr_matrix((golden[stem + "__val"], golden[stem + "__col"],
                          golden[stem + "__rowptr"]), shape=tuple(sh))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def quac():
    import quac_b200 as q
    from quac_b200 import build
    build.build()
    q.lib()
    q.QuaC_initialize()
    return q
