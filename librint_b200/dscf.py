"""Frozen-density gradients with respect to basis exponents and contraction
coefficients -- the reference's python/librint/dscf.py functions (grad, dSf,
dHcoref, dRf, danalyticalf, denergyf) over this library's C ABI.  The result
vector indexes env[s1:s2] as the reference's utils.split does; the adjoint
ERI kernel replaces the Enzyme reverse passes."""
from __future__ import annotations

import numpy as np

from . import _bindings as B
from .basis import Molecule

GRAD_LMAX = 2   # compiled shells on the GPU path


def split(bas) -> tuple[int, int]:
    """env range of the differentiable parameters (src/utils.rs:152-175)."""
    b = np.asarray(bas).reshape(-1, 8)
    s1 = s2 = -1
    for row in b:
        ngto, ex, co = int(row[2]), int(row[5]), int(row[6])
        if s1 == -1 or s1 > ex:
            s1 = ex
        if s2 == -1:
            s2 = co + ngto
        elif s2 < co:
            s2 = co + ngto
    return s1, s2


def _require_grad_domain(m: Molecule):
    b = m.bas.reshape(-1, 8)
    omega = float(m.env[8]) if m.env.size > 8 else 0.0
    if int(b[:, 1].max()) > GRAD_LMAX or omega != 0.0 or int(b[:, 3].max()) > 1:
        raise ValueError("GPU gradient supports shells with l <= 2, nctr == 1 and no range "
                         "separation")


def _call(fname, m: Molecule, P):
    _require_grad_domain(m)
    from .scf import _p2c, _take
    args, _keep = _p2c(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    s1, s2 = split(m.bas)
    ptr = getattr(B.lib(), fname)(*args, P.ctypes.data_as(B.P_d), P.size)
    return _take(ptr, s2 - s1)


def grad(m, P):          # src/p2c.rs:240 -> dH + dR
    return _call("grad_c", m, P)


def dSf(m, P):           # src/p2c.rs:267
    return _call("dS_c", m, P)


def dHcoref(m, P):       # src/p2c.rs:294
    return _call("dHcore_c", m, P)


def dRf(m, P):           # src/p2c.rs:321
    return _call("dR_c", m, P)


def danalyticalf(m, P):  # src/p2c.rs:348 -> dH + dR - dS/2
    return _call("danalytical_c", m, P)


def denergyf(m, P):      # src/p2c.rs:376
    return _call("denergy_c", m, P)
