import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")


@pytest.fixture(scope="session")
def golden_kernels():
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, "kernels_numpy.npz")))


@pytest.fixture(scope="session")
def golden_pipeline():
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, "pipeline_small.npz")))


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle driver (test infrastructure; built on demand)."""
    import subprocess

    lib = os.path.join(ROOT, "oracle", "liboracle_mpr.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    import pipeline

    return pipeline
