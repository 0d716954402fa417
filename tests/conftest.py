"""Test configuration: the `gpu` marker selects tests that need a CUDA device
(B200); everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libbgp.so")


@pytest.fixture(scope="session")
def golden():
    """Fixtures produced by the reference (tests/golden/make_golden.py)."""
    import json
    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")

    def load(name):
        return np.load(os.path.join(d, name + ".npz")), json.load(open(os.path.join(d, name + ".json")))
    return load
