import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    if not os.path.exists(O.LIBORC):
        O.build(ref=False)
    return O


def golden_cases(prefix="levin_ref_"):
    return sorted(os.path.basename(p)[len(prefix):-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def load_golden(name, prefix="levin_ref_"):
    return dict(np.load(os.path.join(GOLDEN, f"{prefix}{name}.npz")))
