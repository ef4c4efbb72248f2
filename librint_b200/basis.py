"""Molecule / basis arrays in librint's (PySCF) layout, without PySCF.

librint takes a molecule as three flat arrays (src/p2c.rs:1-15):

* ``atm``: int32, 6 slots per atom: CHARGE, PTR_COORD, NUC_MOD, PTR_ZETA,
  PTR_FRAC_CHARGE, RESERVE;
* ``bas``: int32, 8 slots per shell: ATOM, ANG, NPRIM, NCTR, KAPPA, PTR_EXP,
  PTR_COEFF, RESERVE;
* ``env``: float64 pool holding coordinates (Bohr), exponents and contraction
  coefficients.  ``env[0]`` overrides the screening cutoff, ``env[8]`` is the
  range-separation omega (must be 0 on this path).  User data starts at
  ``env[20]`` as in PySCF.

Coefficients are stored PySCF-normalised: each primitive carries
``gto_norm(l, a)`` and the contracted function is normalised to one (the
angular factors 1/sqrt(4 pi), sqrt(3/(4 pi)) of s and p shells are applied
inside the integrals, src/g1e.rs:776).  PySCF is not a dependency; the two
normalisation steps are restated here from their definitions.

``read_molecule`` parses the reference's ``molecules/*.txt`` fixture format
(src/utils.rs:17-80), with or without the ``|`` separators.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

ATM_SLOTS = 6
BAS_SLOTS = 8
PTR_ENV_START = 20
BOHR = 0.52917721092          # Angstrom per Bohr (CODATA 2010, as PySCF)


@dataclass
class Molecule:
    atm: np.ndarray
    bas: np.ndarray
    env: np.ndarray
    nelec: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def natm(self) -> int:
        return self.atm.size // ATM_SLOTS

    @property
    def nbas(self) -> int:
        return self.bas.size // BAS_SLOTS

    def nao(self, coord: int = 0) -> int:
        return nao(self.bas, coord)


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int) -> int:
    return 2 * l + 1


def nao(bas: np.ndarray, coord: int = 0) -> int:
    """AO count, nctr included (src/scf.rs:136-151 ``angl``)."""
    b = np.asarray(bas).reshape(-1, BAS_SLOTS)
    return int(sum((ncart(l) if coord == 0 else nsph(l)) * c for l, c in zip(b[:, 1], b[:, 3])))


def gaussian_int(n: int, alpha: float) -> float:
    """int_0^inf x^n exp(-alpha x^2) dx."""
    n1 = (n + 1) * 0.5
    return math.gamma(n1) / (2.0 * alpha ** n1)


def gto_norm(l: int, a: float) -> float:
    """Radial normalisation of r^l exp(-a r^2): 1/sqrt(int r^(2l+2) e^(-2ar^2))."""
    return 1.0 / math.sqrt(gaussian_int(2 * l + 2, 2 * a))


def normalise_contraction(l: int, exps, coefs) -> np.ndarray:
    """PySCF-style stored coefficients for one segmented contraction."""
    exps = np.asarray(exps, dtype=np.float64)
    cs = np.asarray(coefs, dtype=np.float64) * np.array([gto_norm(l, a) for a in exps])
    ee = np.empty((exps.size, exps.size))
    for i, ai in enumerate(exps):
        for j, aj in enumerate(exps):
            ee[i, j] = gaussian_int(2 * l + 2, ai + aj)
    s = float(cs @ ee @ cs)
    return cs / math.sqrt(s)


class Builder:
    """Incremental construction of atm/bas/env."""

    def __init__(self):
        self.atm: list[list[int]] = []
        self.bas: list[list[int]] = []
        self.env: list[float] = [0.0] * PTR_ENV_START
        self.nelec = 0

    def add_atom(self, z: int, xyz_bohr) -> int:
        ptr = len(self.env)
        self.env += [float(v) for v in xyz_bohr]
        self.env.append(0.0)                       # zeta (point nucleus)
        self.atm.append([int(z), ptr, 1, ptr + 3, 0, 0])
        self.nelec += int(z)
        return len(self.atm) - 1

    def add_shell(self, atom: int, l: int, exps, coefs, normalise: bool = True) -> int:
        exps = [float(a) for a in exps]
        cs = normalise_contraction(l, exps, coefs) if normalise else np.asarray(coefs, float)
        pe = len(self.env)
        self.env += exps
        pc = len(self.env)
        self.env += [float(c) for c in cs]
        self.bas.append([atom, l, len(exps), 1, 0, pe, pc, 0])
        return len(self.bas) - 1

    def add_shell_gc(self, atom: int, l: int, exps, coef_sets, normalise: bool = True) -> int:
        """A generally contracted shell: one exponent set, nctr contractions
        (coef_sets[c] over the primitives; each normalised like add_shell).
        env holds the coefficients contraction-major, c[ctr * nprim + prim]
        (libcint's PTR_COEFF layout)."""
        exps = [float(a) for a in exps]
        sets = [normalise_contraction(l, exps, c) if normalise else np.asarray(c, float)
                for c in coef_sets]
        pe = len(self.env)
        self.env += exps
        pc = len(self.env)
        for cs in sets:
            self.env += [float(c) for c in cs]
        self.bas.append([atom, l, len(exps), len(sets), 0, pe, pc, 0])
        return len(self.bas) - 1

    def build(self, name: str = "", **meta) -> Molecule:
        return Molecule(np.array(self.atm, dtype=np.int32).ravel(),
                        np.array(self.bas, dtype=np.int32).ravel(),
                        np.array(self.env, dtype=np.float64), self.nelec, name, dict(meta))


def read_molecule(path: str) -> Molecule:
    """Read a reference ``molecules/*.txt`` fixture (src/utils.rs:17-80)."""
    text = open(path).read()
    if "|" in text:
        parts = text.split("|")
        atm = [int(t) for t in parts[0].split()]
        bas = [int(t) for t in parts[1].split()]
        env = [float(t) for t in " ".join(parts[2:]).split()]
    else:
        atm, bas, env = [], [], []
        for line in text.splitlines():
            toks = line.split()
            if not toks:
                continue
            if all(_is_int(t) for t in toks) and len(toks) == ATM_SLOTS and not bas and not env:
                atm += [int(t) for t in toks]
            elif all(_is_int(t) for t in toks) and len(toks) == BAS_SLOTS and not env:
                bas += [int(t) for t in toks]
            else:
                env += [float(t) for t in toks]
    atm = np.array(atm, dtype=np.int32)
    nel = int(atm.reshape(-1, ATM_SLOTS)[:, 0].sum())
    return Molecule(atm, np.array(bas, dtype=np.int32), np.array(env, dtype=np.float64), nel,
                    name=path)


def _is_int(t: str) -> bool:
    try:
        int(t)
        return True
    except ValueError:
        return False


def shell_offsets(bas: np.ndarray, coord: int = 0) -> np.ndarray:
    b = np.asarray(bas).reshape(-1, BAS_SLOTS)
    dims = [(ncart(l) if coord == 0 else nsph(l)) * c for l, c in zip(b[:, 1], b[:, 3])]
    return np.concatenate([[0], np.cumsum(dims)]).astype(np.int64)
