"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  The product package never does.  ``build()`` runs the
Makefile; ``lib()`` loads oracle/liboracle.so.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_i = ctypes.c_int
_d = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int)
_pd = ctypes.POINTER(ctypes.c_double)
_sz = ctypes.c_size_t


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_rys_roots.argtypes = (_i, _d, _pd, _pd)
        L.orc_set_rys_mode.argtypes = (_i,)
        L.orc_int2e_cart.argtypes = (_pd, _pi, _pi, _i, _pi, _i, _pd)
        L.orc_int2e_cart.restype = _i
        L.orc_int2e_sph.argtypes = (_pd, _pi, _pi, _i, _pi, _i, _pd)
        L.orc_int2e_sph.restype = _i
        L.orc_int2e_batch.argtypes = (_pd, _i, _pi, ctypes.c_long, _pi, _i, _pi, _i, _pd, _i)
        L.orc_int2e_tensor.argtypes = (_pd, _i, _pi, _i, _pi, _i, _pd, _i)
        L.orc_int1e.argtypes = (_pd, _i, _i, _pi, _i, _pi, _i, _pd)
        L.orc_fock_G.argtypes = (_pd, _pd, _i, _pi, _i, _pi, _i, _pd, _i)
        L.orc_density.argtypes = (_pd, _sz, _i, _d, _pi, _i, _pi, _i, _pd, _i, _pi)
        L.orc_density.restype = _i
        L.orc_energy.argtypes = (_pd, _pi, _i, _pi, _i, _pd, _i)
        L.orc_energy.restype = _d
        L.orc_scf.argtypes = (_sz, _i, _d, _pi, _i, _pi, _i, _pd, _i)
        L.orc_scf.restype = _d
        L.orc_fock_G_quartets.argtypes = (_pd, _pd, _pi, ctypes.c_long, _pi, _i, _pi, _i, _pd, _i)
        L.orc_fock_G_blocks.argtypes = (_pd, _pd, _pi, _i, _pi, _i, _pi, _i, _pd, _i)
        L.orc_energy2_sym.argtypes = (_pd, _pi, _i, _pi, _i, _pd, _i)
        L.orc_energy2_sym.restype = _d
        L.orc_energy1.argtypes = (_pd, _pi, _i, _pi, _i, _pd)
        L.orc_energy1.restype = _d
        L.orc_nao.argtypes = (_i, _pi, _i)
        L.orc_nao.restype = _i
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def _mol(m):
    atm = np.ascontiguousarray(m.atm, dtype=np.int32)
    bas = np.ascontiguousarray(m.bas, dtype=np.int32)
    env = np.ascontiguousarray(m.env, dtype=np.float64)
    return atm, bas, env


def rys_roots(n: int, x: float):
    u = np.zeros(n)
    w = np.zeros(n)
    lib().orc_rys_roots(n, float(x), _p(u, _pd), _p(w, _pd))
    return u, w


class independent_roots:
    """Context manager: inside it every Rys rule of the oracle is computed in
    binary128 from the Rys measure itself (orc_set_rys_mode(1): Gauss-
    Legendre discretisation, Stieltjes procedure, Sturm bisection) instead of
    read from the node tables that the CUDA kernels share; about 1 ms per
    rule, for small checks only."""

    def __enter__(self):
        lib().orc_set_rys_mode(1)
        return self

    def __exit__(self, *exc):
        lib().orc_set_rys_mode(0)
        return False


def nao(m, coord=0) -> int:
    _, bas, _ = _mol(m)
    return lib().orc_nao(coord, _p(bas, _pi), bas.size // 8)


def int2e_block(m, shls, coord=1):
    atm, bas, env = _mol(m)
    b = bas.reshape(-1, 8)
    dims = [((b[s, 1] + 1) * (b[s, 1] + 2) // 2 if coord == 0 else 2 * b[s, 1] + 1) * b[s, 3]
            for s in shls]
    out = np.zeros(int(np.prod(dims)))
    sh = np.array(shls, dtype=np.int32)
    f = lib().orc_int2e_cart if coord == 0 else lib().orc_int2e_sph
    nz = f(_p(out, _pd), _p(sh, _pi), _p(atm, _pi), atm.size // 6, _p(bas, _pi), bas.size // 8,
           _p(env, _pd))
    return out.reshape(dims[::-1]).transpose(3, 2, 1, 0), nz


def int2e_batch(m, shls, coord=1, nthreads=0):
    """Packed blocks of many quartets (shls: (nq, 4) int32)."""
    atm, bas, env = _mol(m)
    sh = np.ascontiguousarray(shls, dtype=np.int32)
    b = bas.reshape(-1, 8)
    l = b[:, 1]
    d = ((l + 1) * (l + 2) // 2 if coord == 0 else 2 * l + 1) * b[:, 3]
    total = int(np.prod(d[sh], axis=1).sum())
    out = np.zeros(total)
    lib().orc_int2e_batch(_p(out, _pd), coord, _p(sh, _pi), sh.shape[0], _p(atm, _pi),
                          atm.size // 6, _p(bas, _pi), bas.size // 8, _p(env, _pd), nthreads)
    return out


def int2e_tensor(m, coord=0, nthreads=0):
    atm, bas, env = _mol(m)
    n = nao(m, coord)
    out = np.zeros(n ** 4)
    lib().orc_int2e_tensor(_p(out, _pd), coord, _p(atm, _pi), atm.size // 6, _p(bas, _pi),
                           bas.size // 8, _p(env, _pd), nthreads)
    return out.reshape(n, n, n, n)


def int1e(m, typec, coord=0):
    atm, bas, env = _mol(m)
    n = nao(m, coord)
    out = np.zeros(n * n)
    lib().orc_int1e(_p(out, _pd), coord, typec, _p(atm, _pi), atm.size // 6, _p(bas, _pi),
                    bas.size // 8, _p(env, _pd))
    return out.reshape(n, n)


def fock_G(m, P, coord=0, nthreads=0):
    atm, bas, env = _mol(m)
    n = nao(m, coord)
    P = np.ascontiguousarray(P, dtype=np.float64)
    G = np.zeros(n * n)
    lib().orc_fock_G(_p(G, _pd), _p(P, _pd), coord, _p(atm, _pi), atm.size // 6, _p(bas, _pi),
                     bas.size // 8, _p(env, _pd), nthreads)
    return G.reshape(n, n)


def fock_G_quartets(m, P, shls, nthreads=0):
    """The reference's digestion over the listed quartets only ((nq, 4)
    int32, each visited once as one slot of its nbas^4 loop)."""
    atm, bas, env = _mol(m)
    n = nao(m, 0)
    P = np.ascontiguousarray(P, dtype=np.float64)
    sh = np.ascontiguousarray(shls, dtype=np.int32)
    G = np.zeros(n * n)
    lib().orc_fock_G_quartets(_p(G, _pd), _p(P, _pd), _p(sh, _pi), sh.shape[0], _p(atm, _pi),
                              atm.size // 6, _p(bas, _pi), bas.size // 8, _p(env, _pd), nthreads)
    return G.reshape(n, n)


def fock_G_blocks(m, P, pairs, nthreads=0):
    """G(P) blocks for shell pairs [(X, Y), ...], exact (2 nbas^2 quartets per
    block); returns a list of (nX, nY) arrays."""
    atm, bas, env = _mol(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    b = bas.reshape(-1, 8)
    dims = [(int((b[x, 1] + 1) * (b[x, 1] + 2) // 2), int((b[y, 1] + 1) * (b[y, 1] + 2) // 2))
            for x, y in pr]
    out = np.zeros(sum(a * c for a, c in dims))
    lib().orc_fock_G_blocks(_p(out, _pd), _p(P, _pd), _p(pr, _pi), pr.shape[0], _p(atm, _pi),
                            atm.size // 6, _p(bas, _pi), bas.size // 8, _p(env, _pd), nthreads)
    res, o = [], 0
    for a, c in dims:
        res.append(out[o:o + a * c].reshape(a, c))
        o += a * c
    return res


def energy_sym(m, P, nthreads=0):
    """Energy functional through the unique-quartet two-electron sum."""
    atm, bas, env = _mol(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    a = (_p(P, _pd), _p(atm, _pi), atm.size // 6, _p(bas, _pi), bas.size // 8, _p(env, _pd))
    return lib().orc_energy1(*a) + lib().orc_energy2_sym(*a, nthreads)


def density(m, nelec=None, imax=200, conv=1e-10, nthreads=0):
    atm, bas, env = _mol(m)
    n = nao(m, 0)
    P = np.zeros(n * n)
    it = ctypes.c_int(0)
    rc = lib().orc_density(_p(P, _pd), nelec if nelec is not None else m.nelec, imax, conv,
                           _p(atm, _pi), atm.size // 6, _p(bas, _pi), bas.size // 8,
                           _p(env, _pd), nthreads, ctypes.byref(it))
    if rc != 0:
        raise RuntimeError(f"oracle SCF failed with code {rc} after {it.value} iterations")
    return P.reshape(n, n), it.value


def energy(m, P, nthreads=0):
    atm, bas, env = _mol(m)
    P = np.ascontiguousarray(P, dtype=np.float64)
    return lib().orc_energy(_p(P, _pd), _p(atm, _pi), atm.size // 6, _p(bas, _pi),
                            bas.size // 8, _p(env, _pd), nthreads)


def scf(m, nelec=None, imax=200, conv=1e-10, nthreads=0):
    atm, bas, env = _mol(m)
    return lib().orc_scf(nelec if nelec is not None else m.nelec, imax, conv, _p(atm, _pi),
                         atm.size // 6, _p(bas, _pi), bas.size // 8, _p(env, _pd), nthreads)
