import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_vectors.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libspectral_gpu.so")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def cplx(pairs, dtype=np.complex128):
    a = np.asarray(pairs, dtype=np.float64)
    return (a[:, 0] + 1j * a[:, 1]).astype(dtype)


def test_params(**kw):
    """build_test_sim (src/lib.rs:219-244) as oracle/GPU parameters."""
    from spectral_rs_b200.config import Params
    d = dict(size_x=24, size_y=12, delta=5, dt=0.1, c=3.0, dens=2, gamma_inj=5.0, n_pass=4)
    d.update(kw)
    return Params(**d)


test_params.__test__ = False
