"""CPU tests of the learned-guess host logic and of the network oracle."""
import numpy as np
import pytest

import oracle
from oracle import mlp_ref
from librint_b200 import guess as G
from librint_b200 import synthetic
from librint_b200.basis import Molecule


def _rand_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def _monomials(l, v):
    return np.array([v[0] ** a * v[1] ** b * v[2] ** c for a, b, c in G.cart_exponents(l)])


@pytest.mark.parametrize("l", [0, 1, 2, 3])
def test_cart_rotation_is_function_transform(l):
    rng = np.random.default_rng(l)
    Q = _rand_rotation(rng)
    A = G.cart_rotation(l, Q)
    for _ in range(5):
        v = rng.normal(size=3)
        np.testing.assert_allclose(_monomials(l, Q.T @ v), A @ _monomials(l, v), atol=1e-12)


def test_cart_rotation_representation():
    rng = np.random.default_rng(7)
    Q1, Q2 = _rand_rotation(rng), _rand_rotation(rng)
    for l in range(3):
        np.testing.assert_allclose(G.cart_rotation(l, Q1 @ Q2),
                                   G.cart_rotation(l, Q2) @ G.cart_rotation(l, Q1), atol=1e-12)
        np.testing.assert_allclose(G.cart_rotation(l, Q1.T) @ G.cart_rotation(l, Q1), np.eye(
            (l + 1) * (l + 2) // 2), atol=1e-12)


def _rotated(m: Molecule, Q, shift):
    env = np.array(m.env, dtype=np.float64)
    atm = np.asarray(m.atm).reshape(-1, 6)
    for p in atm[:, 1]:
        env[p:p + 3] = Q @ env[p:p + 3] + shift
    return Molecule(m.atm.copy(), m.bas.copy(), env, m.nelec, m.name + "_rot", {})


def test_density_covariance_and_local_blocks():
    """The oracle's converged density of a rotated molecule is A^T P A, and
    the local-frame blocks and features do not change."""
    m = synthetic.water_like()
    rng = np.random.default_rng(3)
    Q = _rand_rotation(rng)
    mr = _rotated(m, Q, np.array([0.3, -1.2, 2.0]))
    P = oracle.density(m, conv=1e-11)[0]
    Pr = oracle.density(mr, conv=1e-11)[0]
    z, _ = G.molecule_geometry(m)
    lay = G._atom_layout(m)
    n = P.shape[0]
    A = np.zeros((n, n))
    for a, (o, ls, k) in enumerate(lay):
        A[o:o + k, o:o + k] = G.atom_rotation(ls, Q)
    np.testing.assert_allclose(Pr, A.T @ P @ A, atol=2e-8)
    pm = G.PairModel([8, 1], {8: (0, 0, 1), 1: (0,)})     # per-atom exponents differ
    ps, psr = pm.pairs(m), pm.pairs(mr)
    np.testing.assert_allclose(ps.X, psr.X, atol=1e-10)
    y, mk = pm.to_local(m, P, ps)
    yr, _ = pm.to_local(mr, Pr, psr)
    np.testing.assert_allclose(y, yr, atol=2e-8)
    np.testing.assert_allclose(pm.to_density(mr, yr, psr), Pr, atol=2e-8)


def test_local_round_trip_benzene():
    m = synthetic.benzene_like(11)
    pm = G.PairModel.from_molecule(m)
    assert pm.applies(m) and pm.nmax == 15 and pm.ntypes == 5
    rng = np.random.default_rng(0)
    n = m.nao(0)
    P = rng.normal(size=(n, n))
    P = P + P.T
    ps = pm.pairs(m)
    assert len(ps.pairs) == 12 * 13 // 2
    y, mk = pm.to_local(m, P, ps)
    np.testing.assert_allclose(pm.to_density(m, y, ps), P, atol=1e-12)
    # masks: C-C 15x15, C-H 15x5, H-H 5x5
    counts = {int(t): int(mk[ps.types == t][0].sum()) for t in np.unique(ps.types)}
    assert sorted(counts.values()) == [25, 25, 75, 225, 225]


def test_guess_applies_only_to_matching_basis():
    pm = G.PairModel.from_molecule(synthetic.benzene_like(1))
    assert pm.applies(synthetic.benzene_like(2))
    assert not pm.applies(synthetic.water_like())
    assert pm.applies(synthetic.c3_cluster())            # same per-element basis
    assert pm.applies(synthetic.hc_chain())
    assert not pm.applies(synthetic.hc_chain(basis_seed=7))   # another basis draw


def test_mlp_oracle_gradients_vs_finite_differences():
    rng = np.random.default_rng(5)
    sizes = [7, 9, 6, 4]
    params = []
    for k, n in zip(sizes[:-1], sizes[1:]):
        params += [rng.normal(size=(n, k)) / np.sqrt(k), rng.normal(size=n) * 0.1]
    X = rng.normal(size=(5, 7))
    T = rng.normal(size=(5, 4))
    W = (rng.random(size=(5, 4)) > 0.3).astype(float)
    inv = 1.0 / 20
    loss, grads, _ = mlp_ref.loss_and_grad(params, X, T, W, inv)
    h = 1e-6
    for pi, p in enumerate(params):
        flat = p.reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp = mlp_ref.loss_and_grad(params, X, T, W, inv)[0]
            flat[idx] = old - h
            lm = mlp_ref.loss_and_grad(params, X, T, W, inv)[0]
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - grads[pi].reshape(-1)[idx]) < 1e-7 * max(1.0, abs(fd))


def test_adam_oracle_first_step_is_sign_step():
    p = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -0.1, 0.0])
    q, m, v = mlp_ref.adam_step(p, g, np.zeros(3), np.zeros(3), 0.01, 0.9, 0.999, 1e-8, 1)
    np.testing.assert_allclose(q, p - 0.01 * np.array([1.0, -1.0, 0.0]), atol=1e-6)


def test_lowdin_density_round_trip():
    """A converged density survives S^1/2 P S^1/2 and the projection back,
    and a perturbed one comes back idempotent with the right trace."""
    m = synthetic.water_like()
    P = oracle.density(m, conv=1e-11)[0]
    S = oracle.int1e(m, 0)
    Sh, Sih = G.lowdin(S)
    np.testing.assert_allclose(Sh @ Sih, np.eye(len(S)), atol=1e-12)
    Pt = Sh @ P @ Sh
    np.testing.assert_allclose(G.density_from_lowdin(Pt, S, m.nelec // 2), P, atol=1e-9)
    rng = np.random.default_rng(1)
    noise = rng.normal(scale=0.05, size=Pt.shape)
    P0 = G.density_from_lowdin(Pt + noise + noise.T, S, m.nelec // 2)
    assert abs(np.sum(P0 * S) - m.nelec) < 1e-10
    np.testing.assert_allclose(P0 @ S @ P0, 2 * P0, atol=1e-10)


def test_fractional_lowdin_density():
    """The fractional start keeps the electron count, has Loewdin occupations
    in [0, 2] in the order of the predicted eigenvalues, equals the
    projected density for an exact (0 / 2) prediction, and keeps partly
    filled the orbitals a fuzzy prediction leaves near the cut."""
    m = synthetic.water_like()
    P = oracle.density(m, conv=1e-11)[0]
    S = oracle.int1e(m, 0)
    Sh, _ = G.lowdin(S)
    Pt = Sh @ P @ Sh
    np.testing.assert_allclose(G.density_from_lowdin(Pt, S, m.nelec // 2, fractional=True), P,
                               atol=1e-9)
    # a prediction unsure about the 5th and 6th orbitals (7 AOs, 5 occupied)
    _, V = np.linalg.eigh(Pt)
    Pn = (V * np.array([-0.1, 0.2, 0.9, 1.1, 1.9, 2.0, 2.1])) @ V.T
    P0 = G.density_from_lowdin(Pn, S, m.nelec // 2, fractional=True)
    assert abs(np.sum(P0 * S) - m.nelec) < 1e-9
    occ = np.linalg.eigvalsh(Sh @ P0 @ Sh)
    assert occ.min() > -1e-10 and occ.max() < 2 + 1e-10
    assert ((occ > 1e-6) & (occ < 2 - 1e-6)).any()        # some partly filled
    w = np.linalg.eigvalsh(0.5 * (Pn + Pn.T))
    f = G.fractional_occupations(w, m.nelec // 2)
    assert abs(f.sum() - m.nelec) < 1e-9 and (np.diff(f) >= -1e-12).all()


def _pairs_loop(pm, m):
    """Per-pair restatement of PairModel.pairs (frames by _frame), the
    reference for the vectorised version."""
    z, xyz = G.molecule_geometry(m)
    n = len(z)
    nk = len(G.RADIAL_CENTRES)
    out = []
    for a in range(n):
        for b in range(a, n):
            aa, bb = (b, a) if z[b] > z[a] else (a, b)
            t = pm.type_index[(int(z[aa]),)] if aa == bb else pm.type_index[(int(z[aa]), int(z[bb]))]
            o, F = G._frame(xyz, z, aa, bb)
            x = np.zeros(pm.nfeat)
            x[t] = 1.0
            if aa != bb:
                r = np.linalg.norm(xyz[bb] - xyz[aa])
                x[pm.ntypes], x[pm.ntypes + 1] = r, np.exp(-0.5 * r)
            for j in range(n):
                if j in (aa, bb):
                    continue
                d = F @ (xyz[j] - o)
                rj = np.linalg.norm(d)
                g = np.exp(-((rj - G.RADIAL_CENTRES) / G.RADIAL_WIDTH) ** 2)
                blk = pm.ntypes + 2 + pm.elements.index(int(z[j])) * nk * 4
                u = d / max(rj, 1e-12)
                x[blk:blk + nk] += g
                for c in range(3):
                    x[blk + (c + 1) * nk:blk + (c + 2) * nk] += g * u[c]
            out.append(((aa, bb), t, F, x))
    return out


@pytest.mark.parametrize("mol", ["ring", "flake"])
def test_vectorised_pairs_match_loop(mol):
    m = synthetic.benzene_like(21) if mol == "ring" else synthetic.flake_like(20003)
    pm = G.PairModel.from_molecule(synthetic.benzene_like(1))
    ps = pm.pairs(m)
    ref = _pairs_loop(pm, m)
    assert [tuple(p) for p in ps.pairs] == [r[0] for r in ref]
    assert list(ps.types) == [r[1] for r in ref]
    np.testing.assert_allclose(ps.frames, np.array([r[2] for r in ref]), atol=1e-12)
    np.testing.assert_allclose(ps.X, np.array([r[3] for r in ref]), atol=1e-12)
