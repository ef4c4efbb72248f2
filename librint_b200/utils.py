"""The helpers of the reference's python/librint/utils.py over this
package: ``take``, ``prep``, ``pmat``, ``angl``, ``nparams``, ``split``,
``norm`` and ``basis_atm``, with the same arguments and results, so code
written against ``librint.utils`` runs against this library.  ``prep``
takes a PySCF-style molecule or a ``Molecule``; ``norm`` uses this package's
Gaussian integrals instead of PySCF's."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _bindings as B
from .basis import gaussian_int, nao


def take(ptr, shape) -> np.ndarray:
    """Copy a buffer returned by one of the ``*_c`` entry points into numpy
    and release it with ``free_c`` (python/librint/utils.py:9-19)."""
    shape = tuple(int(s) for s in shape)
    n = int(np.prod(shape))
    p = ctypes.cast(ptr, B.P_d)
    out = np.array(np.ctypeslib.as_array(p, shape=shape), copy=True)
    B.lib().free_c(p, n)
    return out


def prep(mol):
    """(atm, bas, env, nelec) of a molecule as contiguous int32 / float64
    arrays, atm (natm, 6) and bas (nbas, 8) (python/librint/utils.py:21-28)."""
    from .scf import as_molecule
    m = as_molecule(mol)
    atm = np.ascontiguousarray(np.asarray(m.atm, dtype=np.int32).reshape(-1, 6))
    bas = np.ascontiguousarray(np.asarray(m.bas, dtype=np.int32).reshape(-1, 8))
    env = np.ascontiguousarray(m.env, dtype=np.float64)
    return atm, bas, env, int(m.nelec)


def pmat(A: np.ndarray):
    """Print a matrix row by row, six decimals, a blank before non-negative
    entries (python/librint/utils.py:30-37)."""
    for row in np.asarray(A):
        print("".join("{:f} ".format(v) if v < 0 else " {:f} ".format(v) for v in row))


def angl(bas: np.ndarray, coord: int = 0) -> int:
    """AO count of ``bas``: cartesian (coord 0) or spherical (1) functions
    per shell times its contractions (python/librint/utils.py:39-48)."""
    return nao(bas, coord)


def nparams(atm, bas, coord: int = 0) -> tuple:
    """(natm, nbas, AO count) (python/librint/utils.py:50-54)."""
    return (len(np.asarray(atm).reshape(-1, 6)), len(np.asarray(bas).reshape(-1, 8)),
            angl(bas, coord))


def split(bas: np.ndarray) -> tuple:
    """env range [s1, s2) of the exponents and coefficients that the
    gradient entry points differentiate (python/librint/utils.py:56-75)."""
    from .dscf import split as _split
    return _split(bas)


def norm(basis_add: list) -> np.ndarray:
    """env entries of shells given as [l, [e, c_1, .., c_nctr], ...]: the
    exponents in descending order, then the coefficients contraction by
    contraction, each contraction scaled so that sum_pq c_p c_q
    int r^(2l+2) e^-(a_p+a_q) r^2 dr = 1 (python/librint/utils.py:77-92;
    no primitive normalisation factor is applied, as there)."""
    env = []
    for b in basis_add:
        l = int(b[0])
        rows = np.array(sorted([list(r) for r in b[1:]], reverse=True), dtype=np.float64)
        es, cs = rows[:, 0], rows[:, 1:]
        ee = np.array([[gaussian_int(2 * l + 2, ai + aj) for aj in es] for ai in es])
        s = np.einsum("pi,pq,qi->i", cs, ee, cs)
        cs = cs / np.sqrt(s)
        env.append(es)
        env.append(cs.T.reshape(-1))
    return np.concatenate(env) if env else np.zeros(0)


def basis_atm(bas: np.ndarray, env: np.ndarray):
    """Renormalise, in place, the coefficients of every segmented shell of
    ``bas`` whose coefficients follow its exponents in ``env`` (the layout
    the reference writes), with ``norm`` (python/librint/utils.py:95-108)."""
    for b in np.asarray(bas).reshape(-1, 8):
        s, b1, b2 = int(b[2]), int(b[5]), int(b[6])
        rows = env[b1:b2 + s].reshape(2, s).T.tolist()
        env[b1:b2 + s] = norm([[int(b[1])] + rows])
