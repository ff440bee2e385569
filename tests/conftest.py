"""Shared test fixtures.

The CPU suite (-m "not gpu") checks the oracle against the reference's
known-answer tests and golden fixtures, the host-side input code, the C ABI
surface (load + exported symbols) and the multi-process host logic.  The GPU
suite (-m gpu) is the parity suite proper: every CUDA result is compared with
the oracle on the same seeded inputs.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_built():
    lib = os.path.join(ROOT, "lumina_b200", "lib", "liblumina_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "lumina_b200", "csrc"), "-j4"],
                       check=True)
    orc = os.path.join(ROOT, "oracle", "liblumina_oracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def backend():
    import lumina_b200 as lb
    return lb.CudaBackend(0)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)


def rand_vec(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
