"""The synthetic systems are the configurations the measurements are quoted
on (no GPU): the water-like system, the ERI sweep's quartet distribution,
the 60-atom C/H cluster of the RHF benchmark, the 20-atom chain of the
gradient checks and the C6H6-like rings of the learned guess, each against
the properties its configuration states (atoms, geometry, shells,
primitives, exponent ranges, AO and electron counts)."""
import numpy as np
import pytest

from librint_b200 import synthetic
from librint_b200.basis import BOHR


def _atoms(m):
    a = m.atm.reshape(-1, 6)
    return a[:, 0], np.array([m.env[p:p + 3] for p in a[:, 1]]) * BOHR


def _shells(m):
    """Per shell: (atom, l, exponents, coefficients)."""
    out = []
    for b in m.bas.reshape(-1, 8):
        k = int(b[2])
        out.append((int(b[0]), int(b[1]), m.env[b[5]:b[5] + k], m.env[b[6]:b[6] + k]))
    return out


def _nearest(a, b, same):
    d = np.linalg.norm(a[:, None] - b[None], axis=-1)
    if same:
        np.fill_diagonal(d, np.inf)
    return d


def test_water_like():
    """O at (0, 0, 0.117) A, H at (0, +-0.757, -0.467) A; shells O s, s, p
    and H s each, 3 primitives, exponents log-uniform in [0.1, 150] sorted
    descending, positive coefficients; 7 AOs, 10 electrons."""
    m = synthetic.water_like()
    z, xyz = _atoms(m)
    assert list(z) == [8, 1, 1]
    np.testing.assert_allclose(xyz, [[0, 0, 0.117], [0, 0.757, -0.467], [0, -0.757, -0.467]],
                               atol=1e-12)
    sh = _shells(m)
    assert [(s[0], s[1]) for s in sh] == [(0, 0), (0, 0), (0, 1), (1, 0), (2, 0)]
    for _, _, e, c in sh:
        assert len(e) == 3 and (e >= 0.1).all() and (e <= 150).all() and (np.diff(e) < 0).all()
        assert (c > 0).all()
    assert m.nao(0) == 7 and m.nelec == 10


@pytest.mark.parametrize("cls", [(0, 0, 0, 0), (2, 1, 1, 0), (2, 2, 2, 2)])
def test_eri_sweep_distribution(cls):
    """Every quartet of the class has its own four shells, each on its own
    centre in a 10 A cube, K uniform in 1..6, exponents log-uniform in
    [0.05, 5000] sorted descending."""
    m, shls = synthetic.eri_sweep(cls, 4000, seed=2)
    z, xyz = _atoms(m)
    sh = _shells(m)
    assert shls.shape == (4000, 4) and len(np.unique(shls)) == 16000
    assert ((xyz >= 0) & (xyz <= 10.0 + 1e-9)).all()
    ls = np.array([s[1] for s in sh]).reshape(-1, 4)
    assert (ls == np.array(cls)).all()
    ks = np.array([len(s[2]) for s in sh])
    assert ks.min() == 1 and ks.max() == 6
    assert abs(ks.mean() - 3.5) < 0.1
    e = np.concatenate([s[2] for s in sh])
    assert e.min() >= 0.05 and e.max() <= 5000
    assert abs(np.log(e).mean() - 0.5 * (np.log(0.05) + np.log(5000))) < 0.1
    assert all((np.diff(s[2]) < 0).all() for s in sh)
    assert len({s[0] for s in sh}) == len(sh)


def test_c3_cluster():
    """60 atoms, 36 C on a perturbed hexagonal lattice (nearest C-C within
    1.40 +- 0.05 A), 24 H at 1.09 +- 0.03 A from an edge carbon; C 3s2p1d and
    H 2s1p with K in 1..6, exponents within C [0.1, 5000] and H [0.1, 50], one
    shell set per element; 288 shells, 660 cartesian AOs, 240 electrons."""
    m = synthetic.c3_cluster()
    z, xyz = _atoms(m)
    C, H = xyz[z == 6], xyz[z == 1]
    assert len(C) == 36 and len(H) == 24
    cc = _nearest(C, C, True)
    nn = cc[cc < 1.7]
    assert nn.min() >= 1.35 and nn.max() <= 1.45
    assert (np.abs(C[:, 2]) < 0.05).all()
    dch = _nearest(H, C, False)
    assert (np.abs(dch.min(axis=1) - 1.09) <= 0.03).all()
    edge = (cc < 1.7).sum(axis=1) < 3
    assert edge[dch.argmin(axis=1)].all()
    sh = _shells(m)
    per = {6: [], 1: []}
    for atom, l, e, c in sh:
        per[int(z[atom])].append((atom, l, tuple(e)))
    assert m.nbas == 288 and m.nao(0) == 660 and m.nelec == 240
    for el, ls, hi in ((6, [0, 0, 0, 1, 1, 2], 5000), (1, [0, 0, 1], 50)):
        rows = per[el]
        atoms = sorted({r[0] for r in rows})
        first = [r[1:] for r in rows if r[0] == atoms[0]]
        assert [f[0] for f in first] == ls
        for a in atoms:                            # the same shells on every atom
            assert [r[1:] for r in rows if r[0] == a] == first
        for l, e in first:
            assert 1 <= len(e) <= 6 and min(e) >= 0.1 and max(e) <= hi


def test_c4_chain():
    """20 atoms (C6H14), C-C 1.54 A and C-H 1.09 A up to the +-0.03 A noise on
    every coordinate, the same per-element basis; 160 cartesian AOs."""
    m = synthetic.hc_chain()
    z, xyz = _atoms(m)
    C, H = xyz[z == 6], xyz[z == 1]
    assert len(C) == 6 and len(H) == 14
    for i in range(5):
        assert abs(np.linalg.norm(C[i + 1] - C[i]) - 1.54) <= 0.03 * 2 * np.sqrt(3)
    assert (np.abs(_nearest(H, C, False).min(axis=1) - 1.09) <= 0.03 * 2 * np.sqrt(3)).all()
    assert m.nao(0) == 160


def test_c5_rings():
    """C6H6-like rings: ring radius (= C-C bond of a regular hexagon)
    1.40 +- 0.05 A, C-H 1.09 +- 0.05 A radially, angles within 3 deg of the
    60-degree steps; 120 cartesian AOs; geometries differ by seed, basis
    does not."""
    for seed in (10000, 10001, 10002):
        m = synthetic.benzene_like(seed)
        z, xyz = _atoms(m)
        C, H = xyz[z == 6], xyz[z == 1]
        r = np.linalg.norm(C, axis=1)
        assert (np.abs(r - 1.40) <= 0.05).all()
        assert (np.abs(np.linalg.norm(H, axis=1) - r - 1.09) <= 0.05).all()
        ang = np.degrees(np.arctan2(C[:, 1], C[:, 0])) % 360
        steps = np.arange(6) * 60.0
        assert (np.abs((ang - steps + 180) % 360 - 180) <= 3.0).all()
        assert m.nao(0) == 120
    a, b = synthetic.benzene_like(10000), synthetic.benzene_like(10001)
    assert not np.allclose(a.env, b.env)
    np.testing.assert_array_equal(a.bas, b.bas)
