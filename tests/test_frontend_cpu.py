"""The Python front end mirrors the reference's python/librint modules: the
same function names, argument order, defaults, string codes and error
behaviour, and it accepts the PySCF-style molecule objects the reference
reads (_atm, _bas, _env, nelec).  Nothing here calls the GPU."""
import inspect
import types

import numpy as np
import pytest

from librint_b200 import dscf, scf, synthetic
from librint_b200.basis import Molecule


def _pyscf_like(m: Molecule):
    return types.SimpleNamespace(_atm=m.atm.reshape(-1, 6).copy(), _bas=m.bas.reshape(-1, 8).copy(),
                                 _env=m.env.copy(), nelec=(m.nelec // 2, m.nelec - m.nelec // 2))


def test_reference_function_names():
    for name in ("int1e", "int2e", "density", "energy", "scf"):
        assert callable(getattr(scf, name))
    for name in ("grad", "dSu", "dSf", "dHcoref", "dRf", "danalyticalf", "denergyf"):
        assert callable(getattr(dscf, name))


def test_reference_argument_order_and_defaults():
    """python/librint/scf.py: int1e(mol, typei='ovlp', coord='cart'),
    int2e(mol, coord='cart'), density(mol, imax=200, conv=1e-6),
    energy(mol, P), scf(mol, imax=200, conv=1e-6)."""
    def head(f, n):
        ps = list(inspect.signature(f).parameters.values())[:n]
        return [(p.name if i else "mol", p.default) for i, p in enumerate(ps)]
    e = inspect.Parameter.empty
    assert head(scf.int1e, 3) == [("mol", e), ("typei", "ovlp"), ("coord", "cart")]
    assert head(scf.int2e, 2) == [("mol", e), ("coord", "cart")]
    assert head(scf.density, 3) == [("mol", e), ("imax", 200), ("conv", 1e-6)]
    assert head(scf.energy, 2) == [("mol", e), ("P", e)]
    assert head(scf.scf, 3) == [("mol", e), ("imax", 200), ("conv", 1e-6)]


def test_pyscf_like_molecule():
    m = synthetic.water_like()
    got = scf.as_molecule(_pyscf_like(m))
    np.testing.assert_array_equal(got.atm, m.atm)
    np.testing.assert_array_equal(got.bas, m.bas)
    np.testing.assert_array_equal(got.env, m.env)
    assert got.nelec == m.nelec == 10
    assert got.atm.dtype == np.int32 and got.env.dtype == np.float64
    assert scf.as_molecule(m) is m
    with pytest.raises(TypeError):
        scf.as_molecule(object())


def test_string_codes_and_reference_messages(capsys):
    """Known codes map to the C ABI's integers (ints pass through); unknown
    strings print the reference's message and return None before any call
    into the library."""
    assert scf._code("nuc", scf.INT1E_TYPES, "") == 2
    assert scf._code("sph", scf.COORDS, "") == 1
    assert scf._code(1, scf.COORDS, "") == 1
    m = synthetic.water_like()
    assert scf.int1e(m, "dipole") is None
    assert "integral type does not exist: ovlp, kin, nuc" in capsys.readouterr().out
    assert scf.int1e(m, "ovlp", "spinor") is None
    assert "coordinate type does not exist: cart, sph" in capsys.readouterr().out
    assert scf.int2e(m, "spinor") is None
    assert "coordinate type does not exist: cart, sph" in capsys.readouterr().out


def test_utils_mirror(capsys):
    """librint_b200.utils follows python/librint/utils.py: AO counts, the
    differentiable env range, per-contraction normalisation of [l, [e, c..]]
    shells (exponents descending, contraction-major coefficients), in-place
    renormalisation of a molecule's shells (a no-op on normalised ones, a
    repair after scaling), prep of a PySCF-style molecule and pmat's format."""
    from librint_b200 import utils
    m = synthetic.water_like()
    assert utils.angl(m.bas.reshape(-1, 8), 0) == m.nao(0) == 7
    assert utils.nparams(m.atm, m.bas) == (3, 5, 7)
    assert utils.split(m.bas) == dscf.split(m.bas)
    env = utils.norm([[1, [0.5, 0.3, 1.0], [4.0, 0.7, 0.0], [1.5, 0.2, 2.0]]])
    e, c = env[:3], env[3:].reshape(2, 3)
    np.testing.assert_array_equal(e, [4.0, 1.5, 0.5])
    from librint_b200.basis import gaussian_int
    ee = np.array([[gaussian_int(4, a + b) for b in e] for a in e])
    np.testing.assert_allclose([ci @ ee @ ci for ci in c], [1.0, 1.0], rtol=1e-14)
    env2 = m.env.copy()
    utils.basis_atm(m.bas.reshape(-1, 8), env2)
    np.testing.assert_allclose(env2, m.env, rtol=1e-13, atol=0)
    b0 = m.bas.reshape(-1, 8)[0]
    env2[b0[6]:b0[6] + b0[2]] *= 2.0
    utils.basis_atm(m.bas.reshape(-1, 8), env2)
    np.testing.assert_allclose(env2, m.env, rtol=1e-13, atol=0)
    atm, bas, env3, nelec = utils.prep(_pyscf_like(m))
    assert atm.shape == (3, 6) and bas.shape == (5, 8) and nelec == 10
    np.testing.assert_array_equal(env3, m.env)
    utils.pmat(np.array([[1.0, -2.0]]))
    assert capsys.readouterr().out == " 1.000000 -2.000000 \n"
