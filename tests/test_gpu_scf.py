"""GPU Fock builds, one-electron integrals and SCF against the oracle and the
reference goldens, through the C ABI."""
import numpy as np
import pytest

import oracle
from librint_b200 import scf, synthetic
from librint_b200.basis import Molecule

pytestmark = pytest.mark.gpu

MOLS = ["h2/sto3g", "lih/sto3g", "hf/sto3g", "h2o/sto3g", "h2o/def2svp", "nh3/sto3g",
        "ch4/sto3g", "c/sto3g", "O/sto3g", "c6h6/sto3g"]


def mol(golden, key):
    return Molecule(golden[key + "/atm"], golden[key + "/bas"], golden[key + "/env"],
                    int(golden[key + "/atm"].reshape(-1, 6)[:, 0].sum()))


@pytest.mark.parametrize("name", MOLS)
def test_int1e_vs_reference(golden, name):
    m = mol(golden, "mol/" + name)
    ctx = scf.MolContext(m)
    for coord in (0, 1):
        for typec in (0, 1, 2):
            np.testing.assert_allclose(ctx.int1e(typec, coord), golden[f"mol/{name}/int1e_{coord}{typec}"],
                                       rtol=1e-12, atol=1e-12)
    # the p2c-shaped entry point too
    np.testing.assert_allclose(scf.int1e(m, 2, 1), golden[f"mol/{name}/int1e_12"], rtol=1e-12,
                               atol=1e-12)


@pytest.mark.parametrize("name", ["h2o/sto3g", "h2o/def2svp", "ch4/sto3g", "c6h6/sto3g"])
def test_fock_G_vs_oracle(golden, name):
    """Direct J/K digestion vs the oracle's integral2e_fock restatement, at a
    random symmetric density and with no screening (tau = 0)."""
    m = mol(golden, "mol/" + name)
    n = m.nao(0)
    rng = np.random.default_rng(1)
    A = rng.standard_normal((n, n))
    P = (A + A.T) / np.sqrt(n)
    G = scf.MolContext(m).fock_G(P, tau=0.0)
    Gr = oracle.fock_G(m, P)
    np.testing.assert_allclose(G, Gr, rtol=1e-11, atol=1e-12 * np.abs(Gr).max())


def test_fock_G_water_like_and_screening(golden):
    m = synthetic.water_like()
    P, _ = oracle.density(m, conv=1e-8)
    ctx = scf.MolContext(m)
    Gr = oracle.fock_G(m, P)
    np.testing.assert_allclose(ctx.fock_G(P, 0.0), Gr, rtol=1e-11, atol=1e-13)
    # screening at 1e-14 changes G by far less than the screening bound
    np.testing.assert_allclose(ctx.fock_G(P, 1e-14), Gr, rtol=0, atol=1e-11)


@pytest.mark.parametrize("name", [n for n in MOLS if n not in ("c6h6/sto3g",)])
def test_scf_reference_algorithm_vs_golden(golden, name):
    """P0 = I, plain Roothaan (the reference's algorithm) -> same fixed point."""
    m = mol(golden, "mol/" + name)
    e = scf.scf(m, imax=1000, conv=1e-10)
    if f"mol/{name}/scf" in golden:
        assert abs(e - golden[f"mol/{name}/scf"]) < 1e-10
    e_orc = oracle.scf(m, conv=1e-10, imax=1000)
    assert abs(e - e_orc) < 1e-10


def test_energy_truths(golden):
    for name, truth in (("h2/sto3g", -0.8817324499460562), ("h2o/sto3g", -74.96102664501196)):
        m = mol(golden, "mol/" + name)
        P = scf.density(m, conv=1e-6, imax=1000)
        assert abs(scf.energy(m, P) - truth) < 1e-10


@pytest.mark.parametrize("name", MOLS)
def test_energy_functional_at_reference_density(golden, name):
    m = mol(golden, "mol/" + name)
    for tag in ("scf", "scf6"):
        if f"mol/{name}/{tag}_P" in golden:
            assert abs(scf.energy(m, golden[f"mol/{name}/{tag}_P"]) - golden[f"mol/{name}/{tag}"]) < 1e-10


def test_diis_core_guess_same_energy(golden):
    """The B200 defaults (core-H guess + DIIS) change iterations, not the energy."""
    for name in ("h2o/def2svp", "c6h6/sto3g", "nh3/sto3g"):
        m = mol(golden, "mol/" + name)
        ctx = scf.MolContext(m)
        r0 = ctx.scf(conv=1e-10, max_iter=1000)
        r1 = ctx.scf(conv=1e-10, guess=1, diis=8)
        assert abs(r0.energy - r1.energy) < 1e-9
        assert r1.iterations <= r0.iterations


def test_water_like_scf(golden):
    m = synthetic.water_like()
    assert abs(scf.scf(m, imax=1000, conv=1e-10) - golden["water_like/scf"]) < 1e-10


def test_scf_failures_in_band(golden):
    """Non-convergence and bad input come back as NaN / exceptions, never a crash."""
    m = mol(golden, "mol/h2o/sto3g")
    assert np.isnan(__import__("librint_b200._bindings", fromlist=["x"]).lib().scf_c(
        *scf._p2c(m)[0], m.nelec, 2, 1e-14))
    with pytest.raises(Exception):
        scf.scf(m, nelec=11)


def _ring():
    return synthetic.benzene_like(seed=10007)


@pytest.mark.parametrize("which", ["ring", "h2o/def2svp"])
def test_fp32_fock_build_error(golden, which):
    """Mixed-precision G(P) against the FP64 build at a converged density:
    all-FP32 quartets stay within 4e-6 of the largest |G| element (per
    element; 1.65e-6 measured on the 120-AO ring, 3.1e-5 absolute at
    max |G| = 18.9, which its tight core shells set) and the split build
    (FP32 only below the bound tau32) within 1e-8."""
    m = _ring() if which == "ring" else Molecule(
        golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
        golden["mol/h2o/def2svp/env"], 10)
    ctx = scf.MolContext(m)
    _, P = ctx.scf(conv=1e-8, guess=1, diis=8, return_density=True)
    G64, n64, z64 = ctx.fock_G_prec(P, 0)
    G32, n32, f32 = ctx.fock_G_prec(P, 1)
    G2, n2, f2 = ctx.fock_G_prec(P, 2, tau32=1e-7)
    ctx.close()
    assert z64 == 0 and f32 == n32 and 0 <= f2 < n2
    e32 = np.abs(G32 - G64).max()
    e2 = np.abs(G2 - G64).max()
    print(f"{which}: FP32 {e32:.3e}, split {e2:.3e} ({f2} of {n2} quartets FP32)")
    assert e32 < 4e-6 * np.abs(G64).max() and e2 < 1e-8


@pytest.mark.parametrize("which", ["ring", "h2o/def2svp"])
def test_mixed_scf_matches_fp64(golden, which):
    """The mixed schedule ends with FP64 builds, so it converges to the FP64
    energy (1e-9 Eh) at the same density threshold, also when its FP32
    phases screen at the looser tau_fp32 the RHF benchmark uses."""
    m = _ring() if which == "ring" else Molecule(
        golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
        golden["mol/h2o/def2svp/env"], 10)
    ctx = scf.MolContext(m)
    r64 = ctx.scf(conv=1e-8, guess=1, diis=8, tau=1e-13)
    rmx = ctx.scf(conv=1e-8, guess=1, diis=8, tau=1e-13, mixed=1)
    rlo = ctx.scf(conv=1e-8, guess=1, diis=8, tau=1e-13, mixed=1, tau_fp32=1e-11)
    ctx.close()
    assert rmx.converged and rmx.fp32_quartets > 0
    assert abs(rmx.energy - r64.energy) < 1e-9, (rmx.energy, r64.energy)
    assert rlo.converged and rlo.quartets <= rmx.quartets
    assert abs(rlo.energy - r64.energy) < 1e-9, (rlo.energy, r64.energy)


@pytest.mark.parametrize("nranks", [2, 3])
def test_fock_partition_shares_sum_to_G(golden, nranks):
    """lrb_fock_G_part: the shares of ranks 0..N-1, computed one after the
    other on this GPU (no rank waits for another), sum to the full G and
    their quartet counts to its count, with and without screening."""
    m = _ring()
    n = m.nao(0)
    rng = np.random.default_rng(4)
    A = rng.standard_normal((n, n))
    P = (A + A.T) / np.sqrt(n)
    ctx = scf.MolContext(m)
    for tau in (0.0, 1e-10):
        G, nq, _ = ctx.fock_G_prec(P, 0, tau=tau)
        parts = [ctx.fock_G_part(P, tau, r, nranks) for r in range(nranks)]
        S = sum(p[0] for p in parts)
        assert sum(p[1] for p in parts) == nq
        assert min(p[1] for p in parts) > 0
        np.testing.assert_allclose(S, G, rtol=1e-12, atol=1e-12 * np.abs(G).max())
    ctx.close()


def test_primitive_screening_error():
    """Primitive-quartet screening (lrb_mol_set_tau_prim) at 1e-15 changes
    G(P) at a converged density by far less than 1e-9 per element, skips
    primitive quartets, and leaves the converged SCF energy within 1e-9 Eh;
    0 restores the reference's primitive set."""
    import ctypes
    from librint_b200 import _bindings as B
    m = _ring()
    ctx = scf.MolContext(m)
    r0, P = ctx.scf(conv=1e-9, guess=1, diis=8, tau=1e-13, return_density=True)
    L = B.lib()
    counts = []
    for tp in (0.0, 1e-15, 0.0):
        ctx.set_tau_prim(tp)
        L.lrb_fock_class_counts((ctypes.c_longlong * 128)(), (ctypes.c_longlong * 128)(), 128)
        L.lrb_profile_enable(1)
        G = ctx.fock_G(P, 1e-13)
        L.lrb_profile_enable(0)
        L.lrb_profile_read((ctypes.c_double * 128)(), 128)
        q, p = (ctypes.c_longlong * 128)(), (ctypes.c_longlong * 128)()
        L.lrb_fock_class_counts(q, p, 128)
        counts.append((G, sum(p)))
    (G0, p0), (G1, p1), (G2, p2) = counts
    print(f"primitive quartets {p0} -> {p1}; max |dG| {np.abs(G1 - G0).max():.3e}")
    assert p1 < p0 and p2 == p0
    assert np.abs(G1 - G0).max() < 1e-9
    assert np.abs(G2 - G0).max() < 1e-12      # atomics order only
    r1 = ctx.scf(conv=1e-9, guess=1, diis=8, tau=1e-13, tau_prim=1e-15)
    ctx.close()
    assert abs(r1.energy - r0.energy) < 1e-9, (r1.energy, r0.energy)


def test_lane_per_primitive_kernels():
    """The lane-per-primitive Fock kernels of the small classes (every such
    quartet routed to them, bound 1) against the slot kernels (bound 1 << 20)
    at tau = 0 (FP64, 1e-12 of max |G|), and both against the oracle's exact
    sums of 12 shell-pair blocks of G (FP64 1e-11; FP32 within the all-FP32
    bound of test_fp32_fock_build_error)."""
    m = _ring()
    ctx = scf.MolContext(m)
    _, P = ctx.scf(conv=1e-8, guess=1, diis=8, return_density=True)
    old = scf.fock_lane_min()
    try:
        res = {}
        for kmin in (1, 1 << 20, 32):
            assert scf.fock_lane_min(kmin) == kmin
            res[kmin] = (ctx.fock_G_prec(P, 0)[0], ctx.fock_G_prec(P, 1)[0])
    finally:
        scf.fock_lane_min(old)
    ctx.close()
    b = m.bas.reshape(-1, 8)
    rng = np.random.default_rng(12)
    pairs = [(int(x), int(y)) for x, y in rng.integers(0, m.nbas, size=(12, 2))]
    ref = oracle.fock_G_blocks(m, P, pairs)
    off = np.concatenate([[0], np.cumsum((b[:, 1] + 1) * (b[:, 1] + 2) // 2)])
    scale = np.abs(res[1 << 20][0]).max()
    bscale = max(np.abs(r).max() for r in ref)
    for kmin, (g64, g32) in res.items():
        e64 = max(np.abs(g64[off[x]:off[x + 1], off[y]:off[y + 1]] - r).max()
                  for (x, y), r in zip(pairs, ref))
        e32 = np.abs(g32 - res[1 << 20][0]).max()
        print(f"lane bound {kmin}: FP64 blocks {e64:.3e} of {bscale:.3e}, FP32 {e32:.3e} of {scale:.3e}")
        assert e64 < 1e-11 * bscale and e32 < 4e-6 * scale
        assert np.abs(g64 - res[1 << 20][0]).max() < 1e-12 * scale
