"""RHF on the GPU: the reference's python/librint/scf.py functions (int1e,
int2e, density, energy, scf) over this library's C ABI, plus a molecule
context for repeated Fock builds."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _bindings as B
from . import eri as _eri
from .basis import Molecule


def _arr(m: Molecule):
    return (np.ascontiguousarray(m.atm, dtype=np.int32), np.ascontiguousarray(m.bas, dtype=np.int32),
            np.ascontiguousarray(m.env, dtype=np.float64))


class MolContext:
    """Device-resident molecule: pair table, Schwarz factors, Fock builds."""

    def __init__(self, m: Molecule):
        self.m = m
        atm, bas, env = _arr(m)
        self._keep = (atm, bas, env)
        h = ctypes.c_void_p()
        rc = B.lib().lrb_mol_create(ctypes.byref(h), atm.ctypes.data_as(B.P_i), atm.size // 6,
                                    bas.ctypes.data_as(B.P_i), bas.size // 8,
                                    env.ctypes.data_as(B.P_d), env.size)
        B.check(rc, "lrb_mol_create")
        self.h = h
        self.nao = B.lib().lrb_mol_nao(h)

    def close(self):
        if self.h:
            B.lib().lrb_mol_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fock_G(self, P, tau: float = 0.0):
        P = np.ascontiguousarray(P, dtype=np.float64)
        G = np.empty_like(P)
        nq = ctypes.c_longlong(0)
        rc = B.lib().lrb_fock_G(self.h, P.ctypes.data_as(B.P_d), G.ctypes.data_as(B.P_d), tau,
                                ctypes.byref(nq))
        B.check(rc, "lrb_fock_G")
        return G

    def set_tau_prim(self, tau_prim: float):
        """Primitive-quartet screening threshold of this context's Fock
        builds (lrb_mol_set_tau_prim; 0 keeps every primitive quartet)."""
        B.check(B.lib().lrb_mol_set_tau_prim(self.h, tau_prim), "lrb_mol_set_tau_prim")

    def fock_G_part(self, P, tau: float, rank: int, nranks: int):
        """This rank's share of G(P) (lrb_fock_G_part); the shares of ranks
        0..nranks-1 sum to fock_G(P, tau).  Returns (G share, quartets)."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        G = np.empty_like(P)
        nq = ctypes.c_longlong(0)
        rc = B.lib().lrb_fock_G_part(self.h, P.ctypes.data_as(B.P_d), G.ctypes.data_as(B.P_d), tau,
                                     rank, nranks, ctypes.byref(nq))
        B.check(rc, "lrb_fock_G_part")
        return G, nq.value

    def fock_G_part_device(self, P, G, tau: float, rank: int, nranks: int, stream=None):
        """Device form: P and G are device tensors (n x n float64, contiguous)
        on the current device; runs on ``stream`` (default: the current
        torch stream)."""
        import torch
        st = torch.cuda.current_stream() if stream is None else stream
        nq = ctypes.c_longlong(0)
        rc = B.lib().lrb_fock_G_part_device(self.h, P.data_ptr(), G.data_ptr(), tau, rank, nranks,
                                            ctypes.byref(nq), ctypes.c_void_p(st.cuda_stream))
        B.check(rc, "lrb_fock_G_part_device")
        return nq.value

    def fock_G_prec(self, P, prec: int, tau: float = 0.0, tau32: float = 0.0):
        """G(P) with the mixed-precision kernels (0 FP64, 1 FP32, 2 FP32 for
        quartets with Schwarz x density bound below tau32); returns
        (G, quartets, fp32 quartets)."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        G = np.empty_like(P)
        nq, n32 = ctypes.c_longlong(0), ctypes.c_longlong(0)
        rc = B.lib().lrb_fock_G_prec(self.h, P.ctypes.data_as(B.P_d), G.ctypes.data_as(B.P_d), tau,
                                     prec, tau32, ctypes.byref(nq), ctypes.byref(n32))
        B.check(rc, "lrb_fock_G_prec")
        return G, nq.value, n32.value

    def int1e(self, typec: int, coord: int = 0):
        n = self.m.nao(coord)
        out = np.empty((n, n))
        B.check(B.lib().lrb_int1e(self.h, typec, coord, out.ctypes.data_as(B.P_d)), "lrb_int1e")
        return out

    def scf(self, nelec=None, max_iter=100, conv=1e-10, guess=0, diis=0, tau=0.0, P0=None,
            return_density=False, mixed=0, fp32_until=1e-3, tau32=1e-7, rebuild_every=6,
            check=True, tau_fp32=0.0, tau_prim=0.0):
        """RHF.  Defaults are the reference's algorithm (P0 = I, plain
        Roothaan, FP64, no screening); guess=1 / diis / tau / mixed select
        the faster schedules, which change iterations and time, not the
        converged energy (mixed: within the tolerance stated in the tests).
        check=False returns a non-converged result (``r.converged`` 0)
        instead of raising.  tau_fp32 (mixed only) is the screening threshold
        of the FP32 and split builds; the FP64 phase screens at tau.
        tau_prim > 0 also skips primitive quartets whose Schwarz x density
        bound is below it (lrb_mol_set_tau_prim) for this SCF's builds."""
        nelec = self.m.nelec if nelec is None else nelec
        o = B.ScfOptions(max_iter, conv, guess, diis, tau, mixed, fp32_until, tau32, rebuild_every,
                         tau_fp32, tau_prim)
        r = B.ScfResult()
        P = np.empty((self.nao, self.nao))
        p0 = None if P0 is None else np.ascontiguousarray(P0, dtype=np.float64).ctypes.data_as(B.P_d)
        rc = B.lib().lrb_scf(self.h, nelec, ctypes.byref(o), ctypes.byref(r),
                             P.ctypes.data_as(B.P_d), p0)
        if check or rc != B.LRB_ERR_SCF:
            B.check(rc, f"lrb_scf ({r.iterations} iterations, delta {r.delta:.3e})")
        return (r, P) if return_density else r

    def energy(self, P, tau: float = 0.0):
        P = np.ascontiguousarray(P, dtype=np.float64)
        E = ctypes.c_double()
        B.check(B.lib().lrb_energy(self.h, P.ctypes.data_as(B.P_d), tau, ctypes.byref(E)), "lrb_energy")
        return E.value


# --- reference python/librint/scf.py shapes (arrays in, arrays out) -------
def fock_lane_min(kmin: int = 0) -> int:
    """Primitive-quartet count from which the small Fock classes run one lane
    per primitive quartet (lrb_fock_lane_min): kmin > 0 sets it for the
    process, 1 << 20 turns those kernels off; returns the value in force."""
    return int(B.lib().lrb_fock_lane_min(int(kmin)))


def _p2c(m: Molecule):
    atm, bas, env = _arr(m)
    return (atm.ctypes.data_as(B.P_i), atm.size, bas.ctypes.data_as(B.P_i), bas.size,
            env.ctypes.data_as(B.P_d), env.size), (atm, bas, env)


def _take(ptr, n):
    if not ptr:
        raise B.LibrintError(B.lib().lrb_last_error().decode() or "NULL result")
    a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
    B.lib().free_c(ptr, n)
    return a


# Codes of the reference's string arguments (python/librint/scf.py:7-36).
INT1E_TYPES = {"ovlp": 0, "kin": 1, "nuc": 2}
COORDS = {"cart": 0, "sph": 1}


def as_molecule(mol) -> Molecule:
    """``mol`` itself when it is a Molecule; otherwise a Molecule from a
    PySCF-style object's ``_atm``, ``_bas``, ``_env`` and ``nelec`` (alpha,
    beta), the fields the reference reads (python/librint/utils.py:21-28)."""
    if isinstance(mol, Molecule):
        return mol
    try:
        atm, bas, env, ne = mol._atm, mol._bas, mol._env, mol.nelec
    except AttributeError as exc:
        raise TypeError("expected a Molecule or an object with _atm, _bas, _env and nelec") from exc
    nelec = int(ne[0] + ne[1]) if np.ndim(ne) else int(ne)
    return Molecule(np.ascontiguousarray(atm, dtype=np.int32).ravel(),
                    np.ascontiguousarray(bas, dtype=np.int32).ravel(),
                    np.ascontiguousarray(env, dtype=np.float64).ravel(), nelec)


def _code(value, table, message):
    """Integer code of a reference string argument (an int passes through);
    None after printing the reference's message for an unknown string."""
    if isinstance(value, str):
        if value not in table:
            print(message)
            return None
        return table[value]
    return int(value)


def int1e(mol, typei="ovlp", coord="cart"):
    """S, T or V (typei 'ovlp' / 'kin' / 'nuc', or 0 / 1 / 2), cartesian or
    spherical (coord 'cart' / 'sph', or 0 / 1): int1e_c, src/p2c.rs:86.
    Unknown strings print the reference's message and return None."""
    typec = _code(typei, INT1E_TYPES, "integral type does not exist: ovlp, kin, nuc")
    if typec is None:
        return None
    c = _code(coord, COORDS, "coordinate type does not exist: cart, sph")
    if c is None:
        return None
    m = as_molecule(mol)
    args, _keep = _p2c(m)
    n = m.nao(c)
    return _take(B.lib().int1e_c(*args, c, typec), n * n).reshape(n, n)


def int2e(mol, coord="cart"):
    """The dense (n, n, n, n) ERI tensor (int2e_c, src/p2c.rs:109; the
    reference's integral2e layout, src/scf.rs:215)."""
    c = _code(coord, COORDS, "coordinate type does not exist: cart, sph")
    if c is None:
        return None
    return _eri.int2e(as_molecule(mol), c)


def density(mol, imax: int = 200, conv: float = 1e-6, nelec=None):
    """Converged density (density_c, src/p2c.rs:153); RuntimeError
    (LibrintError) when the SCF fails.  nelec defaults to the molecule's."""
    m = as_molecule(mol)
    args, _keep = _p2c(m)
    n = m.nao(0)
    nelec = m.nelec if nelec is None else nelec
    return _take(B.lib().density_c(*args, nelec, imax, conv), n * n).reshape(n, n)


def energy(mol, P):
    """Total energy at the density P (energy_c, src/p2c.rs:186)."""
    m = as_molecule(mol)
    args, _keep = _p2c(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    e = B.lib().energy_c(*args, P.ctypes.data_as(B.P_d), P.size)
    if np.isnan(e):
        raise B.LibrintError(B.lib().lrb_last_error().decode())
    return e


def scf(mol, imax: int = 200, conv: float = 1e-6, nelec=None):
    """Converged RHF energy (scf_c, src/p2c.rs:210); RuntimeError
    (LibrintError) when the SCF fails.  nelec defaults to the molecule's."""
    m = as_molecule(mol)
    args, _keep = _p2c(m)
    nelec = m.nelec if nelec is None else nelec
    e = B.lib().scf_c(*args, nelec, imax, conv)
    if np.isnan(e):
        raise B.LibrintError(B.lib().lrb_last_error().decode())
    return e
