"""f shells (the one-CTA-per-quartet kernels of eri_gen.cu) and generally
contracted shells (split into segmented sub-shells on the host) on the GPU,
against the oracle and the reference's own vectors
(tests/golden/make_golden_fgc.py)."""
import numpy as np
import pytest

import oracle
from librint_b200 import eri, scf, synthetic
from tests.conftest import (ERI_ATOL, ERI_RTOL, assert_block_close_or_exact,
                            assert_close_block_scale, assert_eri_close, cart_block_scale, f_classes,
                            fgc_molecule)

pytestmark = pytest.mark.gpu


def _block(m, shls, coord):
    """One quartet through the batch path, as an [i, j, k, l] array."""
    b = np.asarray(m.bas).reshape(-1, 8)
    d = [((b[s, 1] + 1) * (b[s, 1] + 2) // 2 if coord == 0 else 2 * b[s, 1] + 1) * b[s, 3]
         for s in shls]
    out = eri.int2e_batch(m, np.array([shls], dtype=np.int32), coord)
    return out.reshape(d[::-1]).transpose(3, 2, 1, 0)


@pytest.mark.parametrize("cls", f_classes(), ids=lambda c: "%d%d%d%d" % c)
def test_f_class_samples(golden_fgc, cls):
    """The reference's three compact quartets of the class: cartesian blocks
    against the oracle (40-digit arbiter where they differ), spherical
    blocks at 1e-12 relative plus 1e-12 of the cartesian scale."""
    for q in range(3):
        key = "f/%d%d%d%d/%d" % (cls + (q,))
        m = fgc_molecule(golden_fgc, key)
        got = _block(m, [0, 1, 2, 3], 0)
        ref, _ = oracle.int2e_block(m, [0, 1, 2, 3], 0)
        assert_block_close_or_exact(got, ref, m, [0, 1, 2, 3], what=key)
        scale = np.abs(ref).max()
        got = _block(m, [0, 1, 2, 3], 1)
        ref, _ = oracle.int2e_block(m, [0, 1, 2, 3], 1)
        assert (np.abs(got - ref) <= 1e-12 * np.abs(ref) + 1e-12 * scale + 1e-15).all(), key
        # and the reference's own block, at the same spherical bar
        want = golden_fgc[f"{key}/sph"]
        assert (np.abs(got - want) <= 1e-12 * np.abs(want) + 1e-12 * scale + 1e-15).all(), key


@pytest.mark.parametrize("cls", f_classes(), ids=lambda c: "%d%d%d%d" % c)
def test_f_sweep_vs_oracle(cls):
    """300 quartets per f class, compact sweep distribution (centres in a
    2.5 A cube, K = 1..4, exponents log-uniform in [0.1, 50]), cartesian and
    spherical, against the oracle: 1e-12 relative per integral plus 2e-11 of
    its quartet's largest cartesian element plus 5e-15 (spherical elements
    are sums of cartesian ones, and their rounding scales with those).  The small elements of these
    blocks come out of cancellation in the horizontal recurrences, and
    against 40-digit values both FP64 paths err by far more than 1e-12 of
    the block scale there; so the elements outside the bar must be within
    5e-9 of their quartet's largest cartesian element (1e-7 for (ff|ff);
    30x that for spherical elements, each a sum of up to 4^4 cartesian ones
    with coefficients up to ~2.5 per shell), and the two
    quartets with the largest excess go to the 40-digit arbiter (GPU no
    further from it than 4x the oracle, or 1e-11 of the block scale).
    Measured on the 97 quartets this bar flags in (ff|dd) .. (ff|ff) (seed
    31), cartesian blocks against 40-digit values: largest GPU error 7.0e-10
    of the block scale outside (ff|ff) ((ff|fd), 3.5e-15 absolute on a scale
    of 5.0e-6; the oracle's 4.5e-10), the oracle's largest 5.7e-10; in
    (ff|ff) GPU 3.8e-8 and oracle 3.6e-8 (a quartet where both err by
    1.6e-11 absolute); largest GPU - oracle difference 8.5e-10 of the block
    scale outside (ff|ff) and 2.4e-8 in it."""
    m, shls = synthetic.eri_sweep(cls, 300, seed=31, kmax=4, cube_ang=2.5, elo=0.1, ehi=50.0)
    done = set()
    cart = oracle.int2e_batch(m, shls, 0)
    for coord in (0, 1):
        got = eri.int2e_batch(m, shls, coord)
        ref = oracle.int2e_batch(m, shls, coord)
        assert_close_block_scale(got, ref, m, shls, coord, rel_block=2e-11,
                                 scale_values=cart_block_scale(m, shls, coord, cart),
                                 rel_hard=(1e-7 if cls == (3, 3, 3, 3) else 5e-9) * (1 if coord == 0 else 30),
                                 atol=5e-15, max_arbitrated=2, arbitrated=done,
                                 what=f"f sweep {cls} coord {coord}",
                                 gpu_cart=lambda sh: eri.int2e_batch(m, sh, 0))


@pytest.mark.parametrize("key", ["gc", "fpol"])
def test_gc_and_f_molecules(golden_fgc, key):
    """Generally contracted (O s x2, p x3, H s x2) and f-polarised water:
    int1e against the reference, the dense int2e_c tensor against the
    oracle per integral, the energy functional at the reference's density
    (1e-10 Eh), G(P) against the oracle's nbas^4 digestion (tau = 0)."""
    g = golden_fgc
    m = fgc_molecule(g, key)
    for coord in (0, 1):
        for typec in (0, 1, 2):
            np.testing.assert_allclose(scf.int1e(m, typec, coord), g[f"{key}/int1e_{coord}{typec}"],
                                       rtol=1e-12, atol=1e-12)
        assert_eri_close(eri.int2e(m, coord).ravel(), oracle.int2e_tensor(m, coord).ravel(),
                         what=f"{key} int2e_c coord {coord}")
    P = g[f"{key}/scf_P"]
    assert abs(scf.energy(m, P) - float(g[f"{key}/scf"])) < 1e-10
    ctx = scf.MolContext(m)
    Gr = oracle.fock_G(m, P)
    np.testing.assert_allclose(ctx.fock_G(P, 0.0), Gr, rtol=1e-11, atol=1e-12 * np.abs(Gr).max())
    r, Pg = ctx.scf(conv=1e-10, guess=1, diis=8, return_density=True)
    ctx.close()
    # the GPU's fixed point: its energy is the oracle's functional there
    assert abs(r.energy - oracle.energy(m, Pg)) < 1e-10
    if key == "fpol":       # the reference, the oracle and the GPU share this fixed point
        assert abs(r.energy - float(g["fpol/scf"])) < 1e-9


def test_gc_libcint_per_quartet(golden_fgc):
    """int2e_sph / int2e_cart on quartets of generally contracted shells
    (blocks of nf * nctr rows per shell, contraction-major) against the
    oracle's per-quartet blocks."""
    m = fgc_molecule(golden_fgc, "gc")
    for shls in ([0, 1, 0, 1], [1, 1, 3, 4], [0, 3, 2, 1], [4, 4, 4, 4]):
        for coord in (0, 1):
            ref, _ = oracle.int2e_block(m, shls, coord)
            got, nz = eri.int2e_block(m, shls, coord)
            assert nz == 1
            err = np.abs(got - ref)
            assert (err <= ERI_RTOL * np.abs(ref) + ERI_ATOL).all(), (shls, coord, err.max())


def test_gc_batch_matches_split_shells(golden_fgc):
    """lrb_int2e_batch on generally contracted shells equals the blocks of
    the same molecule with every contraction as its own segmented shell,
    reassembled (the split is exact up to the screening coefficient)."""
    from tests.conftest import segmented_copy
    m = fgc_molecule(golden_fgc, "gc")
    rng = np.random.default_rng(8)
    shls = rng.integers(0, m.nbas, size=(200, 4)).astype(np.int32)
    got = eri.int2e_batch(m, shls, 1)
    ref = oracle.int2e_batch(m, shls, 1)
    assert_eri_close(got, ref, what="gc batch")
    ms, _ = segmented_copy(m)
    assert ms.nbas > m.nbas
