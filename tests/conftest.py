import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.npz")
GOLDEN_FGC = os.path.join(ROOT, "tests", "golden", "reference_fgc.npz")

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


@pytest.fixture(scope="session")
def golden_fgc():
    """f-shell and general-contraction vectors from the reference's shipped
    library (tests/golden/make_golden_fgc.py)."""
    import numpy as np
    return np.load(GOLDEN_FGC)


def fgc_molecule(g, key):
    from librint_b200.basis import Molecule
    atm = g[key + "/atm"]
    return Molecule(atm, g[key + "/bas"], g[key + "/env"], int(atm.reshape(-1, 6)[:, 0].sum()))


def f_classes():
    from librint_b200 import synthetic
    return [c for c in synthetic.canonical_classes(3) if max(c) == 3]


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


def segmented_copy(m):
    """The molecule with every generally contracted shell split into its
    contractions (consecutive segmented shells, same AO order) and, per AO,
    its (segmented shell, cartesian component)."""
    import numpy as np
    from librint_b200.basis import Molecule
    b = np.asarray(m.bas).reshape(-1, 8)
    nb, ao = [], []
    for row in b:
        l, k, nc = int(row[1]), int(row[2]), int(row[3])
        for c in range(nc):
            nb.append([row[0], l, k, 1, 0, row[5], row[6] + c * k, 0])
            ao += [(len(nb) - 1, comp) for comp in range((l + 1) * (l + 2) // 2)]
    return Molecule(m.atm, np.array(nb, dtype=np.int32).ravel(), m.env, m.nelec), ao


def assert_cart_elements_close_or_exact(got, ref, m, idx, what="", max_elements=64):
    """Sampled elements (flat indices into the n^4 cartesian tensor) against
    ref at the per-integral tolerance; where they differ, a 40-digit
    evaluation (oracle/mp_exact.py, generally contracted shells split)
    decides: got may not be further from it than 4x ref's error + 1e-15."""
    import numpy as np
    from oracle import mp_exact
    got, ref = np.asarray(got), np.asarray(ref)
    bad = np.nonzero(np.abs(got - ref) > ERI_RTOL * np.abs(ref) + ERI_ATOL)[0]
    assert len(bad) <= max_elements, f"{what}: {len(bad)} elements outside tolerance"
    if not len(bad):
        return
    ms, ao = segmented_copy(m)
    n = len(ao)
    bs = np.asarray(ms.bas).reshape(-1, 8)
    for e in bad:
        a, b, c, d = np.unravel_index(int(idx[e]), (n, n, n, n))
        sh = [ao[a][0], ao[b][0], ao[c][0], ao[d][0]]
        comp = [ao[a][1], ao[b][1], ao[c][1], ao[d][1]]
        nf = [(bs[s, 1] + 1) * (bs[s, 1] + 2) // 2 for s in sh]
        ex = mp_exact.eri_cart_exact(ms.atm, ms.bas, ms.env, sh)
        v = ex[comp[0] + nf[0] * (comp[1] + nf[1] * (comp[2] + nf[2] * comp[3]))]
        assert abs(got[e] - v) <= 4.0 * abs(ref[e] - v) + ERI_ATOL, \
            f"{what} element {idx[e]}: error {abs(got[e] - v):.3e} vs exact, reference's {abs(ref[e] - v):.3e}"


def assert_block_close_or_exact(got, ref, m, shls, what=""):
    """One cartesian quartet block (libcint layout, i fastest, as an array
    indexed [i, j, k, l]) against ref, arbitrated element-wise by the
    40-digit evaluation where the two differ beyond the tolerance."""
    import numpy as np
    from oracle import mp_exact
    got, ref = np.asarray(got), np.asarray(ref)
    bad = np.abs(got - ref) > ERI_RTOL * np.abs(ref) + ERI_ATOL
    if not bad.any():
        return
    ex = np.asarray(mp_exact.eri_cart_exact(m.atm, m.bas, m.env, list(shls))).reshape(
        ref.shape[::-1]).transpose(3, 2, 1, 0)
    assert (np.abs(got - ex)[bad] <= 4.0 * np.abs(ref - ex)[bad] + ERI_ATOL).all(), \
        f"{what}: further from the 40-digit value than the reference"


def block_scale(m, shls, coord, values):
    """Per element, the largest |value| of the quartet block it belongs to
    (packed libcint blocks of the quartet list ``shls``)."""
    import numpy as np
    off = np.concatenate([[0], np.cumsum(_block_sizes(m, shls, coord))])
    v = np.abs(np.asarray(values))
    mx = np.maximum.reduceat(v, off[:-1]) if v.size else v
    return np.repeat(mx, np.diff(off))


def cart_block_scale(m, shls, coord, cart_values):
    """Per element of the ``coord`` layout of the quartet list ``shls``, the
    largest |value| of the same quartet's cartesian block (``cart_values``,
    packed cartesian blocks of the same list): the magnitude the spherical
    transform's rounding scales with."""
    import numpy as np
    mx = block_scale(m, shls, 0, cart_values)
    off0 = np.concatenate([[0], np.cumsum(_block_sizes(m, shls, 0))])
    per_q = mx[off0[:-1]] if len(off0) > 1 else mx
    return np.repeat(per_q, _block_sizes(m, shls, coord))


def assert_close_block_scale(got, ref, m, shls, coord, scale_values=None, rel_block=1e-12,
                             what="", atol=ERI_ATOL, gpu_cart=None, max_arbitrated=3,
                             rel_hard=None, exact_floor=1e-11, arbitrated=None):
    """Per integral 1e-12 relative plus ``rel_block`` of the largest |value| of
    its quartet block (of ``scale_values``, default ref) plus ``atol``: the
    bar for blocks whose small elements come out of cancellation between
    much larger terms (high-momentum blocks; short range as full minus long
    range).  Elements outside it must still be within ``rel_hard`` of the
    block scale (when given; else none may be outside), and the worst
    ``max_arbitrated`` quartets among them (largest difference over block
    scale; cartesian blocks from ``gpu_cart(shls)``) go to the 40-digit
    evaluation: the GPU may not be further from it than 4x the oracle's error,
    or ``exact_floor`` of the exact block's largest element, plus 1e-15.
    ``arbitrated`` (a set) carries the quartets already judged across calls
    on the same quartet list (cartesian and spherical passes)."""
    import numpy as np
    got, ref = np.asarray(got), np.asarray(ref)
    scale = block_scale(m, shls, coord, ref if scale_values is None else scale_values)
    diff = np.abs(got - ref)
    bad = diff > ERI_RTOL * np.abs(ref) + rel_block * scale + atol
    if not bad.any():
        return
    rel = diff / np.maximum(scale, 1e-300)
    off = np.concatenate([[0], np.cumsum(_block_sizes(m, shls, coord))])
    owner = np.searchsorted(off, np.nonzero(bad)[0], side="right") - 1
    quartets = np.unique(owner)
    msg = (f"{what}: {bad.sum()} of {bad.size} outside in {len(quartets)} quartets; flagged "
           f"elements: largest |diff| {diff[bad].max():.3e}, largest |diff| / block scale "
           f"{rel[bad].max():.3e}")
    print(msg)
    if gpu_cart is None:
        raise AssertionError(msg)
    if rel_hard is None:
        assert len(quartets) <= max_arbitrated, msg
    else:
        assert (diff[bad] <= ERI_RTOL * np.abs(ref[bad]) + rel_hard * scale[bad] + atol).all(), \
            msg + f" (beyond {rel_hard:g} of the block scale)"
    worst = {}
    for q, r in zip(owner, rel[bad]):
        worst[q] = max(worst.get(q, 0.0), r)
    import oracle
    from oracle import mp_exact
    for q in sorted(worst, key=lambda k: -worst[k])[:max_arbitrated]:
        if arbitrated is not None:
            if q in arbitrated:
                continue
            arbitrated.add(q)
        sh = np.ascontiguousarray(np.asarray(shls)[q:q + 1], dtype=np.int32)
        ex = np.array(mp_exact.eri_cart_exact(m.atm, m.bas, m.env, sh[0]), dtype=float).ravel()
        e_or = np.abs(oracle.int2e_batch(m, sh, 0) - ex).max()
        e_gpu = np.abs(gpu_cart(sh) - ex).max()
        assert e_gpu <= max(4.0 * e_or, exact_floor * np.abs(ex).max()) + ERI_ATOL, \
            f"{what} quartet {q}: GPU error vs exact {e_gpu:.3e}, oracle's {e_or:.3e}"


