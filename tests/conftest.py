import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "be_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libbe_b200.so")


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN) as z:
        data = {k: z[k] for k in z.files}
    cases = {}
    for k, v in data.items():
        dim, name, field = k.split("/")
        cases.setdefault((dim, name), {})[field] = v
    return cases


@pytest.fixture(scope="session")
def ctx():
    import labeling_b200 as be
    c = be.Context(0)
    yield c
    c.close()
