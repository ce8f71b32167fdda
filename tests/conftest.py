"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and run the engine's kernels;
everything else runs on the CPU (oracle pins, host logic, ABI surface, gloo multi-process)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine's kernels")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "reference_vectors.npz")))


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference library (oracle/_ref) not built on this machine")
    return Reference()


@pytest.fixture(scope="session")
def sim():
    from openqarp_b200 import B200Simulator
    s = B200Simulator()
    yield s
    s.close()


@pytest.fixture(scope="session")
def sim64():
    from openqarp_b200 import B200Simulator
    s = B200Simulator(dtype="complex64")
    yield s
    s.close()


def masks_from(golden, prefix):
    from openqarp_b200.observable import PauliMasks
    return PauliMasks(golden[prefix + "_obs_x"], golden[prefix + "_obs_z"], golden[prefix + "_obs_c"])


class Stream:
    """A packed stream rebuilt from golden arrays (same fields as ir.PackedStream)."""

    def __init__(self, golden, prefix):
        self.buf = golden[prefix + "_buf"].tobytes()
        self.dep_ptr = golden[prefix + "_dep_ptr"].astype(np.int32)
        self.dep_param = golden[prefix + "_dep_param"].astype(np.int32)
        self.dep_alpha = golden[prefix + "_dep_alpha"].astype(np.float64)
