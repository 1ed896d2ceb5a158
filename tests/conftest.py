import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


def load_hbuild_case(name):
    z = np.load(os.path.join(GOLDEN, "hbuild_ref.npz"))
    pre = name + "__"
    return {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}


def hbuild_case_names():
    z = np.load(os.path.join(GOLDEN, "hbuild_ref.npz"))
    return sorted({k.split("__")[0] for k in z.files})


def upper_to_full(upper, nb):
    """Column-major upper triangle (as stored in the fixtures) to a symmetric nb x nb array."""
    M = np.zeros((nb, nb))
    iu = np.triu_indices(nb)
    M[iu] = upper
    return M + np.triu(M, 1).T


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle
