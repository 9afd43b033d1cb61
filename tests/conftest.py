import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def pytest_collection_modifyitems(config, items):
    # every test ends within 15 minutes: a test that never returns (a CPU
    # oracle stuck in C code, say) ends the run instead of holding it (the
    # thread method also stops code that never returns to Python)
    for item in items:
        if item.get_closest_marker("timeout") is None:
            item.add_marker(pytest.mark.timeout(900, method="thread"))


@pytest.fixture(scope="session")
def b200():
    import libgrid_b200

    return libgrid_b200.load()


@pytest.fixture(scope="session")
def restate():
    from oracle import pyoracle

    return pyoracle.restatement()


@pytest.fixture(scope="session")
def ref():
    from oracle import pyoracle

    if not pyoracle.reference_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    return pyoracle.reference(min(8, os.cpu_count() or 1))


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
