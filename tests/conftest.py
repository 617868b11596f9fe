import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import bindings  # noqa: E402  (test infrastructure)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle():
    if not bindings.port_available():
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "port"], stdout=subprocess.DEVNULL)
    if not bindings.ref_available():  # built only where the recipe finds the reference sources
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref-if-present"], stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def port():
    _ensure_oracle()
    return bindings.PortLib()


@pytest.fixture(scope="session")
def ref():
    _ensure_oracle()
    if not bindings.ref_available():
        pytest.skip("compiled reference oracle (oracle/_ref) not available")
    return bindings.RefLib()


@pytest.fixture(scope="session")
def engine():
    import shockhash_b200 as shg
    return shg.Engine(0)


def rand_u64(rng, n):
    return rng.integers(0, 2**64, size=n, dtype=np.uint64)


def unique_u64(rng, n):
    a = np.unique(rand_u64(rng, n + 16))
    while len(a) < n:
        a = np.unique(np.concatenate([a, rand_u64(rng, n)]))
    rng.shuffle(a)
    return a[:n]
