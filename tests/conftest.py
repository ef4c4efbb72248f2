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


def _block_sizes(m, shls, coord):
    import numpy as np
    bas = np.asarray(m.bas).reshape(-1, 8)
    l = bas[np.asarray(shls), 1]
    n = (l + 1) * (l + 2) // 2 if coord == 0 else 2 * l + 1
    return n.prod(axis=1)


def assert_eri_close_or_exact(got, ref, m, shls, coord, gpu_cart, what="", max_quartets=10):
    """Per-integral tolerance against the oracle; where the two disagree beyond
    it, a 40-digit evaluation of the quartet (oracle/mp_exact.py, cartesian)
    decides: the GPU block may not be further from it than 4x the oracle's
    own error plus 1e-15.  Some quartets with distant centres and wide
    exponent ranges lose digits to cancellation in the reference's own
    recurrences, so there the oracle is not an exact target either.
    ``gpu_cart(shls)`` returns the GPU's cartesian blocks for a quartet list."""
    import numpy as np
    import oracle
    from oracle import mp_exact
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape, (what, got.shape, ref.shape)
    err = np.abs(got - ref)
    bad = err > ERI_RTOL * np.abs(ref) + ERI_ATOL
    if not bad.any():
        return
    off = np.concatenate([[0], np.cumsum(_block_sizes(m, shls, coord))])
    quartets = np.unique(np.searchsorted(off, np.nonzero(bad)[0], side="right") - 1)
    assert len(quartets) <= max_quartets, \
        f"{what}: {bad.sum()} elements in {len(quartets)} quartets outside tolerance"
    for q in quartets:
        sh = np.ascontiguousarray(np.asarray(shls)[q:q + 1], dtype=np.int32)
        ex = np.array(mp_exact.eri_cart_exact(m.atm, m.bas, m.env, sh[0]), dtype=float).ravel()
        o = oracle.int2e_batch(m, sh, 0)
        g = gpu_cart(sh)
        e_or, e_gpu = np.abs(o - ex).max(), np.abs(g - ex).max()
        assert e_gpu <= 4.0 * e_or + ERI_ATOL, \
            f"{what} quartet {q}: GPU error vs exact {e_gpu:.3e}, oracle's {e_or:.3e}"
