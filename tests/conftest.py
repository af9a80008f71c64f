import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def golden():
    """dict case -> arrays recorded from the reference (tests/golden/make_golden.py)."""
    out = {}
    for f in sorted(os.listdir(GOLDEN)):
        if f.endswith(".npz"):
            with np.load(os.path.join(GOLDEN, f)) as z:
                out[f[:-4]] = {k: z[k] for k in z.files}
    return out
