"""Frozen-density gradients with respect to basis exponents and contraction
coefficients -- the reference's python/librint/dscf.py functions (grad, dSf,
dHcoref, dRf, danalyticalf, denergyf; each takes a Molecule or a PySCF-style
object, like the scf module) over this library's C ABI.  The result
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


def _call(fname, mol, P):
    from .scf import _p2c, _take, as_molecule
    m = as_molecule(mol)
    _require_grad_domain(m)
    args, _keep = _p2c(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    s1, s2 = split(m.bas)
    ptr = getattr(B.lib(), fname)(*args, P.ctypes.data_as(B.P_d), P.size)
    return _take(ptr, s2 - s1)


def dSu(mol) -> np.ndarray:
    """Overlap Jacobian (s2 - s1, n, n): [l, nu, mu] = d S[mu nu] / d env[s1 + l]
    (src/p2c.rs:131; the reference's python/librint/dscf.py dSu layout)."""
    from .scf import _p2c, _take, as_molecule
    m = as_molecule(mol)
    _require_grad_domain(m)
    args, _keep = _p2c(m)
    s1, s2 = split(m.bas)
    n = m.nao(0)
    return _take(B.lib().dS_u(*args), n * n * (s2 - s1)).reshape(n, n, s2 - s1).transpose(2, 0, 1)


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


# ---------------------------------------------------------------- coordinates
def nuclear_gradient(m: Molecule, P, tau: float = 0.0) -> np.ndarray:
    """dE/dR (natm, 3) of the RHF energy at a converged density P: this
    library's extension to coordinates (the reference differentiates only
    env[s1:s2]).  One-electron centre derivatives with the Hellmann-Feynman
    term, -1/2 sum (P F P) dS, the adjoint ERI kernel's centre derivatives
    and the nuclear repulsion."""
    _require_grad_domain(m)
    from .scf import MolContext
    ctx = MolContext(m)
    try:
        P = np.ascontiguousarray(P, dtype=np.float64)
        out = np.empty(3 * m.natm)
        B.check(B.lib().lrb_grad_nuc(ctx.h, P.ctypes.data_as(B.P_d), tau,
                                     out.ctypes.data_as(B.P_d)), "lrb_grad_nuc")
    finally:
        ctx.close()
    return out.reshape(m.natm, 3)


def int1e_jacobian(m: Molecule, typec: int) -> np.ndarray:
    """(n*n, nenv) Jacobian of S (0), T (1) or V (2) with respect to all of
    env; row nu*n + mu, the layout of the reference's Enzyme checks."""
    from .scf import MolContext
    ctx = MolContext(m)
    try:
        n = ctx.nao
        out = np.empty(n * n * m.env.size)
        B.check(B.lib().lrb_int1e_jacobian(ctx.h, typec, out.ctypes.data_as(B.P_d)),
                "lrb_int1e_jacobian")
    finally:
        ctx.close()
    return out.reshape(n * n, m.env.size)


def with_coordinates(m: Molecule, xyz) -> Molecule:
    """Copy of m with the atoms at xyz (natm, 3) Bohr."""
    env = np.array(m.env, dtype=np.float64)
    atm = np.asarray(m.atm).reshape(-1, 6)
    for a, p in enumerate(atm[:, 1]):
        env[p:p + 3] = np.asarray(xyz, dtype=np.float64)[a]
    return Molecule(m.atm.copy(), m.bas.copy(), env, m.nelec, m.name, dict(m.meta))


def with_parameters(m: Molecule, theta) -> Molecule:
    """Copy of m with env[s1:s2] (exponents and coefficients) replaced."""
    env = np.array(m.env, dtype=np.float64)
    s1, s2 = split(m.bas)
    env[s1:s2] = np.asarray(theta, dtype=np.float64)
    return Molecule(m.atm.copy(), m.bas.copy(), env, m.nelec, m.name, dict(m.meta))


def coordinates(m: Molecule) -> np.ndarray:
    atm = np.asarray(m.atm).reshape(-1, 6)
    return np.stack([np.asarray(m.env)[p:p + 3] for p in atm[:, 1]])


_SCF_DEFAULTS = dict(conv=1e-10, guess=1, diis=8, max_iter=200)


def _energy_and_density(m: Molecule, scf_kwargs):
    from .scf import MolContext
    ctx = MolContext(m)
    try:
        r, P = ctx.scf(return_density=True, **dict(_SCF_DEFAULTS, **(scf_kwargs or {})))
    finally:
        ctx.close()
    return r.energy, P


def _torch_function():
    import torch

    class RHFEnergy(torch.autograd.Function):
        """E(coordinates, env[s1:s2]) of converged RHF on the GPU; the backward
        pass uses lrb_grad_nuc for the coordinates and danalytical (dH + dR -
        dS/2) for the basis parameters, both at the converged density."""

        @staticmethod
        def forward(ctx, xyz, theta, mol, scf_kwargs):
            m = with_parameters(with_coordinates(mol, xyz.detach().cpu().numpy()),
                                theta.detach().cpu().numpy())
            e, P = _energy_and_density(m, scf_kwargs)
            ctx.mol, ctx.P = m, P
            return torch.tensor(e, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            gx = gt = None
            if ctx.needs_input_grad[0]:
                gx = g * torch.from_numpy(nuclear_gradient(ctx.mol, ctx.P))
            if ctx.needs_input_grad[1]:
                gt = g * torch.from_numpy(danalyticalf(ctx.mol, ctx.P))
            return gx, gt, None, None

    return RHFEnergy


def rhf_energy(mol: Molecule, xyz, theta=None, scf_kwargs=None):
    """Differentiable RHF energy: ``xyz`` (natm, 3) and optional ``theta``
    (env[s1:s2]) are torch tensors; the result is a 0-d float64 tensor whose
    backward gives dE/dR and dE/dtheta."""
    import torch
    if theta is None:
        s1, s2 = split(mol.bas)
        theta = torch.tensor(np.asarray(mol.env)[s1:s2])
    return _torch_function().apply(xyz, theta, mol, scf_kwargs)
