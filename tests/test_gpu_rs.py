"""Range-separated ERIs (env[8] = omega) on the GPU against the oracle:
dense tensors, sweep quartets and Fock builds for omega > 0 (long range,
erf(omega r)/r) and omega < 0 (short range, erfc(|omega| r)/r).  The oracle
is pinned to the reference's vectors and, where the reference's own
short-range nodes fail (Rys order >= 4), to 40-digit evaluations
(tests/test_oracle_pins.py)."""
import numpy as np
import pytest

import oracle
from librint_b200 import eri, scf, synthetic
from librint_b200.basis import Molecule
from tests.conftest import assert_close_block_scale, assert_eri_close, fgc_molecule

pytestmark = pytest.mark.gpu


def _with_omega(m, omega):
    env = np.array(m.env, dtype=np.float64)
    env[8] = omega
    return Molecule(m.atm, m.bas, env, m.nelec)


@pytest.mark.parametrize("omega", [0.3, -0.3, -2.0])
def test_dense_tensors(golden, omega):
    svp = Molecule(golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
                   golden["mol/h2o/def2svp/env"], 10)
    for m in (synthetic.water_like(), svp):
        mo = _with_omega(m, omega)
        for coord in (0, 1):
            assert_eri_close(eri.int2e(mo, coord).ravel(), oracle.int2e_tensor(mo, coord).ravel(),
                             what=f"omega {omega} coord {coord}")


@pytest.mark.parametrize("omega", [0.5, -0.5])
@pytest.mark.parametrize("cls", [(0, 0, 0, 0), (1, 1, 1, 0), (2, 1, 1, 1), (2, 2, 2, 2), (3, 1, 2, 0)],
                         ids=lambda c: "%d%d%d%d" % c if isinstance(c, tuple) else str(c))
def test_sweep_classes(omega, cls):
    """500 quartets per class of a compact sweep distribution (centres in a
    4 A cube, K = 1..4), spherical, against the oracle: 1e-12 relative per
    integral plus 2e-11 of the largest element of the quartet's block under
    the full operator.  Short range is the full integral minus the
    long-range one, and the recurrences of compact high-momentum blocks
    amplify rounding: against 40-digit values both paths err by up to ~5e-15
    absolute on (dd|dd) blocks (long range, scale 3e-4: GPU 5.4e-15, oracle
    4.0e-15; short range, scale 2e-8: GPU 3.2e-15, oracle 3.4e-15), hence
    the 5e-15 floor; quartets beyond it go to the 40-digit arbiter."""
    m0, shls = synthetic.eri_sweep(cls, 500, seed=41, kmax=4, cube_ang=4.0, elo=0.1, ehi=200.0)
    m = _with_omega(m0, omega)
    got = eri.int2e_batch(m, shls, 1)
    ref = oracle.int2e_batch(m, shls, 1)
    full = oracle.int2e_batch(m0, shls, 1)
    assert_close_block_scale(got, ref, m, shls, 1, scale_values=np.maximum(np.abs(full), np.abs(ref)),
                             rel_block=2e-11, atol=5e-15, what=f"omega {omega} {cls}",
                             gpu_cart=lambda sh: eri.int2e_batch(m, sh, 0))


@pytest.mark.parametrize("omega", [0.4, -0.4])
def test_fock_build_and_energy(golden_fgc, omega):
    """G(P) with the attenuated operator against the oracle's nbas^4
    digestion (tau = 0), and the converged SCF energy equals the oracle's
    energy functional at the GPU's density (f shells included)."""
    m = _with_omega(fgc_molecule(golden_fgc, "fpol"), omega)
    n = m.nao(0)
    rng = np.random.default_rng(12)
    A = rng.standard_normal((n, n))
    P = (A + A.T) / np.sqrt(n)
    ctx = scf.MolContext(m)
    Gr = oracle.fock_G(m, P)
    np.testing.assert_allclose(ctx.fock_G(P, 0.0), Gr, rtol=1e-11, atol=1e-12 * np.abs(Gr).max())
    r, Pg = ctx.scf(conv=1e-10, guess=1, diis=8, return_density=True, max_iter=300)
    ctx.close()
    assert abs(r.energy - oracle.energy(m, Pg)) < 1e-10
