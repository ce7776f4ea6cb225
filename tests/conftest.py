"""Shared test configuration.

Markers: ``gpu`` — needs a CUDA device (run with ``-m gpu``); everything else
runs on the CPU.  The oracle under oracle/ is imported here only as the checker.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "lightning-unification_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


# Tolerances: complex128 results match the FP64 oracle to 1e-12; complex64
# results (FP32 amplitudes, FP32-pair compensated gate arithmetic, FP64
# reductions) to the stated bound below.
TOL = {np.complex128: 1e-12, np.complex64: 2e-6}


@pytest.fixture(scope="session")
def ref_module():
    import ref
    m = ref.load()
    if m is None:
        pytest.skip("oracle/_ref not built (make -C oracle)")
    return m


def random_state(rng, n, dtype=np.complex128):
    s = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    s /= np.linalg.norm(s)
    return s.astype(dtype)
