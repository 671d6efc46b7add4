import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def restated():
    from oracle.oracle import Restated
    return Restated()


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    here = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(here, "manifest.json")) as f:
        manifest = json.load(f)["cases"]
    arrays = dict(np.load(os.path.join(here, "golden.npz")))
    return manifest, arrays
