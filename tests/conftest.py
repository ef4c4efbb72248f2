import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.npz")

# Per-integral tolerance used throughout: relative 1e-12 with an absolute floor
# of 1e-15 Hartree.  Below ~1e-20 both the reference and the oracle lose
# relative accuracy to cancellation (triangulated against 40-digit mpmath by
# oracle/mp_exact.py), so a purely relative bar is not meaningful there.
ERI_RTOL = 1e-12
ERI_ATOL = 1e-15


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(GOLDEN)


def assert_eri_close(got, ref, rtol=ERI_RTOL, atol=ERI_ATOL, what=""):
    import numpy as np
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape, (what, got.shape, ref.shape)
    err = np.abs(got - ref)
    bound = rtol * np.abs(ref) + atol
    bad = err > bound
    if bad.any():
        i = np.argmax(err - bound)
        raise AssertionError(f"{what}: {bad.sum()} of {err.size} outside tolerance; worst "
                             f"got={got.flat[i]!r} ref={ref.flat[i]!r} err={err.flat[i]:.3e}")
