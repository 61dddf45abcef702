"""Shared fixtures. Marker ``gpu``: needs a CUDA device (B200) and the built library; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "palmtracer-cpp_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GAUSS_PARAMS = np.array([7.0, 1.0, 2.0, 0.0])  # Tests_CPU/test_Palm.cpp:25


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built sm_100a library")


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import OracleLib, ORACLE_SO
    if not os.path.exists(ORACLE_SO):
        import subprocess
        subprocess.check_call(["bash", os.path.join(ROOT, "oracle", "build_oracle.sh")])
    return OracleLib()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import reference
    return reference()


@pytest.fixture(scope="session")
def stacks():
    return np.load(os.path.join(GOLDEN, "stacks.npz"))


@pytest.fixture(scope="session")
def goldens():
    return np.load(os.path.join(GOLDEN, "localizations.npz"))


@pytest.fixture(scope="session")
def lib():
    """The product library; a GPU test fails (never skips) when it cannot be loaded."""
    import ptb
    return ptb
