import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "cc-fjpy_b200"), os.path.join(REPO, "oracle"),
          os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(REPO, "tests", "golden", "reference_outputs.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def lib():
    from ccfj import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def probe():
    """The test-only special-function probe library (not the product)."""
    from ccfj import _lib
    return _lib.load_probe()
