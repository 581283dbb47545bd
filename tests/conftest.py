import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def restated():
    import oracle
    return oracle.restated()


@pytest.fixture(scope="session")
def ref_lib():
    import oracle
    if not oracle.RefIndex.available():
        if os.path.isdir(os.path.join(oracle.REFERENCE_SRC, "src")):
            oracle.build(reference=True)
        else:
            pytest.skip("reference oracle library not built and reference sources absent")
    oracle.RefIndex.set_threads(0)
    return oracle.RefIndex


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_ivf.npz"))
