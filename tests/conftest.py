import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# reference checkout (read only), present in the build container only
REFERENCE_DIR = os.environ.get("SCC_REFERENCE_DIR", "/root/reference")
SAMPLES = ["sample0", "sample4", "sample5", "sample1", "sample128", "sample2"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: full-size configurations")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(n) for n in SAMPLES}


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def native():
    from detectingscc_b200 import _native
    from detectingscc_b200 import build as b
    if not os.path.exists(_native.LIB_PATH):
        b.build()
    return _native
