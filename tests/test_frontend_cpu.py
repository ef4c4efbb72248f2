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
