"""Seeded synthetic molecules for the workloads this library is measured on.

No public dataset is involved: every input is drawn from the stated
distributions with ``numpy.random.default_rng(seed)``.  Coordinates are given
in Angstrom and stored in Bohr; exponents are sorted descending (PySCF order);
contraction coefficients are positive and PySCF-normalised
(``basis.normalise_contraction``).

* ``water_like``     -- O at (0,0,0.117) A, H at (0,+-0.757,-0.467) A;
  shells O: s,s,p and H: s; 3 primitives each, exponents log-uniform
  in [0.1, 150]; 5 shells, 7 AOs, 10 electrons.
* ``eri_sweep``      -- independent shell quartets of one angular class; every
  shell has its own centre (uniform in a 10 A cube), K uniform in 1..6 and
  exponents log-uniform in [0.05, 5000].
* ``ch_basis``       -- the C/H basis every C/H system below uses: one shell
  set per element drawn from seed 3 (C 3s2p1d, H 2s1p, K uniform in 1..6,
  exponents log-uniform within each shell's core / valence / diffuse /
  polarisation range, together C [0.1, 5000] and H [0.1, 50]).
* ``c3_cluster``     -- the 60-atom RHF system: 36 C on a perturbed hexagonal
  lattice (C-C 1.40 +- 0.05 A) and 24 H at 1.09 A on edge carbons,
  660 cartesian AOs.
* ``hc_cluster``     -- the same flake construction for any carbon count.
* ``hc_chain``       -- zig-zag C_nH_(2n+2) chain, C-C 1.54 A, C-H 1.09 A,
  +-0.03 A noise (n = 6: 20 atoms).
* ``flake_like``     -- hc_cluster construction with 8..20 carbons, for
  training the learned guess on flake environments.
* ``benzene_like``   -- C6H6 ring, bonds +-0.05 A, angles +-3 deg.
"""
from __future__ import annotations

import math

import numpy as np

from .basis import BOHR, Builder, Molecule, normalise_contraction

ANG2BOHR = 1.0 / BOHR


def _exps(rng, k, lo, hi):
    e = np.exp(rng.uniform(math.log(lo), math.log(hi), size=k))
    return np.sort(e)[::-1]


def _coefs(rng, k):
    return rng.uniform(0.2, 1.0, size=k)


def water_like(seed: int = 1) -> Molecule:
    rng = np.random.default_rng(seed)
    b = Builder()
    o = b.add_atom(8, np.array([0.0, 0.0, 0.117]) * ANG2BOHR)
    h1 = b.add_atom(1, np.array([0.0, 0.757, -0.467]) * ANG2BOHR)
    h2 = b.add_atom(1, np.array([0.0, -0.757, -0.467]) * ANG2BOHR)
    for atom, l in ((o, 0), (o, 0), (o, 1), (h1, 0), (h2, 0)):
        b.add_shell(atom, l, _exps(rng, 3, 0.1, 150.0), _coefs(rng, 3))
    return b.build("water_like", seed=seed)


# canonical classes li>=lj, lk>=ll, (li,lj)>=(lk,ll) for l in {s,p,d}
def canonical_classes(lmax: int = 2):
    pairs = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    return [(p[0], p[1], q[0], q[1]) for i, p in enumerate(pairs) for q in pairs[: i + 1]]


def eri_sweep(cls, nq: int, seed: int = 2, kmax: int = 6, cube_ang: float = 10.0,
              elo: float = 0.05, ehi: float = 5000.0) -> tuple[Molecule, np.ndarray]:
    """One angular class: nq independent quartets, one atom per shell.

    Returns the molecule arrays and shls (nq, 4) int32.  Vectorised; the
    stream of random numbers depends on (seed, cls, nq) only.
    """
    li = np.array(cls, dtype=np.int64)
    rng = np.random.default_rng([seed] + list(cls))
    nsh = 4 * nq
    ls = np.tile(li, nq)
    ks = rng.integers(1, kmax + 1, size=nsh)
    xyz = rng.uniform(0.0, cube_ang, size=(nsh, 3)) * ANG2BOHR
    raw_e = np.exp(rng.uniform(math.log(elo), math.log(ehi), size=(nsh, kmax)))
    raw_c = rng.uniform(0.2, 1.0, size=(nsh, kmax))
    mask = np.arange(kmax)[None, :] < ks[:, None]
    e = np.where(mask, raw_e, -np.inf)
    order = np.argsort(-e, axis=1)
    e = np.take_along_axis(e, order, axis=1)
    c = np.take_along_axis(np.where(mask, raw_c, 0.0), order, axis=1)
    e = np.where(mask, e, 0.0)
    cn = np.empty_like(c)
    step = 1 << 17
    for a in range(0, nsh, step):
        cn[a:a + step] = _normalise_many(ls[a:a + step], e[a:a + step], c[a:a + step],
                                         mask[a:a + step])
    # env: 20 reserved, then per shell [x y z 0 | exps(K) | coefs(K)]
    per = 4 + 2 * ks
    start = 20 + np.concatenate([[0], np.cumsum(per)[:-1]])
    env = np.zeros(20 + int(per.sum()))
    env[start[:, None] + np.arange(3)[None, :]] = xyz
    cols = np.arange(kmax)[None, :]
    pe = start + 4
    pc = pe + ks
    env[(pe[:, None] + cols)[mask]] = e[mask]
    env[(pc[:, None] + cols)[mask]] = cn[mask]
    atm = np.zeros((nsh, 6), dtype=np.int32)
    atm[:, 1] = start
    atm[:, 2] = 1
    atm[:, 3] = start + 3
    bas = np.zeros((nsh, 8), dtype=np.int32)
    bas[:, 0] = np.arange(nsh)
    bas[:, 1] = ls
    bas[:, 2] = ks
    bas[:, 3] = 1
    bas[:, 5] = pe
    bas[:, 6] = pc
    shls = np.arange(nsh, dtype=np.int32).reshape(nq, 4)
    mol = Molecule(atm.ravel(), bas.ravel(), env, 0, f"eri_sweep{cls}",
                   {"seed": seed, "class": tuple(int(v) for v in cls)})
    return mol, shls


def _normalise_many(ls, e, c, mask):
    """Vectorised normalise_contraction over shells (rows)."""
    gtab = np.array([math.gamma(l + 1.5) for l in range(9)])
    gam = gtab[ls][:, None]
    n1 = (ls[:, None] + 1.5).astype(np.float64)
    # gto_norm(l, a) = 1/sqrt(gamma(l+3/2)/(2 (2a)^(l+3/2)))
    with np.errstate(divide="ignore", invalid="ignore"):
        nrm = np.where(mask, 1.0 / np.sqrt(gam / (2.0 * (2.0 * np.where(mask, e, 1.0)) ** n1)), 0.0)
    cs = c * nrm
    a = np.where(mask, e, 1.0)
    s = a[:, :, None] + a[:, None, :]
    ee = gam[:, :, None] / (2.0 * s ** n1[:, :, None])
    ee = np.where(mask[:, :, None] & mask[:, None, :], ee, 0.0)
    tot = np.einsum("si,sij,sj->s", cs, ee, cs)
    return cs / np.sqrt(tot)[:, None]


# ------------------------------------------------------------------ C/H sets
# A split-valence set with polarisation ("DZP-like"): C 3s2p1d, H 2s1p.  Each
# shell has a role -- core, valence, diffuse or polarisation -- and draws K
# uniform in 1..6 and its exponents log-uniform within its role's range; the
# ranges span C [0.1, 5000] and H [0.1, 50].  Drawing every shell over the
# whole range instead makes every contracted function tight (the smallest
# kinetic-energy diagonal of the 120-AO ring was 7.8 Eh and its
# core-Hamiltonian HOMO +11.5 Eh) and no SCF converges on such a set.
C_ROLES = ((0, 3.0, 5000.0),    # s core
           (0, 0.25, 5.0),      # s valence
           (0, 0.1, 0.3),       # s diffuse
           (1, 0.3, 30.0),      # p valence
           (1, 0.1, 0.4),       # p diffuse
           (2, 0.3, 2.0))       # d polarisation
H_ROLES = ((0, 0.3, 50.0),      # s valence
           (0, 0.1, 0.3),       # s diffuse
           (1, 0.3, 2.0))       # p polarisation
CH_BASIS_SEED = 3               # the one basis every C/H system here uses


def _draw_shells(rng, z, kmax):
    out = []
    for l, lo, hi in (C_ROLES if z == 6 else H_ROLES):
        k = int(rng.integers(1, kmax + 1))
        out.append((l, _exps(rng, k, lo, hi), _coefs(rng, k)))
    return out


def ch_basis(seed: int = CH_BASIS_SEED, kmax: int = 6) -> dict:
    """One shell set per element, like a named basis: C 3s2p1d, H 2s1p, K
    uniform in 1..kmax per shell, exponents log-uniform within each shell's
    role range (C_ROLES, H_ROLES), coefficients uniform in [0.2, 1]
    (normalised when the shell is added).  C is drawn first, then H, from
    default_rng(seed)."""
    rng = np.random.default_rng(seed)
    return {z: _draw_shells(rng, z, kmax) for z in (6, 1)}


def _build_ch(z, xyz_ang, name, basis_seed=CH_BASIS_SEED, **meta):
    b = Builder()
    for zi, r in zip(z, xyz_ang):
        b.add_atom(zi, np.asarray(r) * ANG2BOHR)
    table = ch_basis(basis_seed)
    for atom, zi in enumerate(z):
        for l, e, c in table[zi]:
            b.add_shell(atom, l, e, c)
    return b.build(name, basis_seed=basis_seed, **meta)


def _honeycomb(a=1.40, n=10):
    pts = []
    for i in range(-n, n + 1):
        for j in range(-n, n + 1):
            o = np.array([i * 1.5 * a, (i + 2 * j) * math.sqrt(3) / 2 * a])
            pts.append(o + np.array([a / 2, 0.0]))
            pts.append(o + np.array([-a / 2, 0.0]))
    return np.unique(np.round(np.array(pts), 6), axis=0)


def _flake(rng, ncarbon, aspect, theta_deg=0.0, shift=(0.0, 0.0)):
    """C/H flake geometry (Angstrom): the ``ncarbon`` honeycomb sites
    (C-C 1.40 A) nearest ``shift`` in the metric sqrt(x'^2 + (aspect y')^2)
    of axes rotated by theta_deg (an elongated flake, so enough edge sites
    carry H); one H at 1.09 A on each carbon with two carbon neighbours, two
    (tilted out of plane) on each carbon with one; carbons perturbed by
    +-0.05 A in bond length.  Returns (Z list, xyz)."""
    a = 1.40
    pts = _honeycomb(a)
    t = math.radians(theta_deg)
    rot = np.array([[math.cos(t), -math.sin(t)], [math.sin(t), math.cos(t)]])
    q = (pts - np.asarray(shift)) @ rot.T
    d = np.sqrt(q[:, 0] ** 2 + (aspect * q[:, 1]) ** 2)
    c2 = pts[np.argsort(d, kind="stable")[:ncarbon]]
    hs = []
    tilt = math.radians(54.75)
    for p in c2:
        nb = [x for x in c2 if 0.1 < np.linalg.norm(x - p) < 1.1 * a]
        if len(nb) >= 3 or not nb:
            continue
        v = -sum((x - p) / np.linalg.norm(x - p) for x in nb)
        v = np.append(v / np.linalg.norm(v), 0.0)
        p3 = np.append(p, 0.0)
        if len(nb) == 2:
            hs.append(p3 + 1.09 * v)
        else:
            for sz in (1.0, -1.0):
                hs.append(p3 + 1.09 * (math.cos(tilt) * v + sz * math.sin(tilt) * np.array([0, 0, 1.0])))
    c3 = np.column_stack([c2, np.zeros(len(c2))])
    c3 += rng.uniform(-0.05, 0.05, size=c3.shape) / math.sqrt(3)
    return [6] * len(c3) + [1] * len(hs), np.vstack([c3, np.array(hs)])


def c3_cluster(seed: int = 3) -> Molecule:
    """The ~600-AO RHF system: 60-atom C/H flake, 36 C + 24 H (240
    electrons), C on a perturbed hexagonal lattice (1.40 +- 0.05 A), H at
    1.09 A on edge carbons, the seed-3 per-element basis (C 3s2p1d, H 2s1p,
    K = 1..6, log-uniform exponents per shell role): 288 shells, 660
    cartesian AOs."""
    z, xyz = _flake(np.random.default_rng(seed), 36, 3.0, 10.0, (0.35, 0.0))
    return _build_ch(z, xyz, "c3_cluster", seed=seed)


def hc_cluster(seed: int = 3, ncarbon: int = 34, aspect: float = 2.0) -> Molecule:
    """Flake of ``ncarbon`` carbons (``_flake`` with the metric unrotated),
    the per-element basis."""
    z, xyz = _flake(np.random.default_rng(seed), ncarbon, aspect)
    return _build_ch(z, xyz, "hc_cluster", seed=seed)


def flake_like(seed: int) -> Molecule:
    """A small closed-shell C/H flake for training the learned guess: the
    hc_cluster construction with 8..20 carbons and aspect 1..2.5 drawn from
    ``seed`` (carbons added until the electron count is even)."""
    g = np.random.default_rng([seed, 77])
    nc = int(g.integers(8, 21))
    aspect = float(g.uniform(1.0, 2.5))
    while True:
        m = hc_cluster(seed=seed, ncarbon=nc, aspect=aspect)
        if m.nelec % 2 == 0:
            m.name = "flake_like"
            m.meta = {"seed": seed, "ncarbon": nc, "aspect": aspect}
            return m
        nc += 1


def hc_chain(seed: int = 4, ncarbon: int = 6, basis_seed: int = CH_BASIS_SEED) -> Molecule:
    """Zig-zag C_nH_(2n+2) chain (C-C 1.54 A, C-H 1.09 A, +-0.03 A noise on
    every coordinate); n = 6 gives the 20-atom chain (160 cartesian AOs)."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.54, 1.09
    ang = math.radians(109.47)
    cs = []
    for i in range(ncarbon):
        cs.append([i * cc * math.sin(ang / 2), (i % 2) * cc * math.cos(ang / 2), 0.0])
    cs = np.array(cs)
    hs = []
    for i, p in enumerate(cs):
        up = 1.0 if i % 2 else -1.0
        for sz in (1.0, -1.0):
            v = np.array([0.0, up * math.cos(ang / 2), sz * math.sin(ang / 2)])
            hs.append(p + ch * v / np.linalg.norm(v))
        if i in (0, ncarbon - 1):
            v = np.array([-1.0 if i == 0 else 1.0, up * 0.3, 0.0])
            hs.append(p + ch * v / np.linalg.norm(v))
    xyz = np.vstack([cs, np.array(hs)])
    xyz += rng.uniform(-0.03, 0.03, size=xyz.shape)
    z = [6] * ncarbon + [1] * len(hs)
    return _build_ch(z, xyz, "hc_chain", basis_seed=basis_seed, seed=seed)


def benzene_like(seed: int = 5, basis_seed: int = CH_BASIS_SEED) -> Molecule:
    """One C6H6-like ring; geometry from ``seed`` (bonds +-0.05 A, angles
    +-3 deg); basis: the per-element set drawn from ``basis_seed`` (C
    3s2p1d = 15, H 2s1p = 5 cartesian AOs; 120 AOs in all)."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.40, 1.09
    cs, hs = [], []
    for i in range(6):
        t = math.radians(60 * i + rng.uniform(-3, 3))
        r = (cc + rng.uniform(-0.05, 0.05))
        cs.append([r * math.cos(t), r * math.sin(t), 0.0])
        rh = r + ch + rng.uniform(-0.05, 0.05)
        hs.append([rh * math.cos(t), rh * math.sin(t), 0.0])
    xyz = np.vstack([cs, hs])
    return _build_ch([6] * 6 + [1] * 6, xyz, "benzene_like", basis_seed=basis_seed, seed=seed)
