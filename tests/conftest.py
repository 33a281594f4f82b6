"""Shared test set-up: the `gpu` marker, the import path, and built artefacts.

`-m "not gpu"` runs the oracle-vs-golden, host-build and ABI tests on the CPU;
`-m gpu` runs the parity tests through the C ABI on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session", autouse=True)
def _built():
    # Build only what is missing: the prebuilt libraries travel with the tree.
    from oracle import oracle
    if not os.path.exists(oracle._LIB_PATH):
        oracle.build(force=True)
    from rapidfem_b200 import build as nb
    if not os.path.exists(nb.LIB):
        nb.build(force=True)
    yield


def rel_l2(got, want):
    import numpy as np
    got = np.asarray(got, dtype=np.float64).ravel()
    want = np.asarray(want, dtype=np.float64).ravel()
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300))
