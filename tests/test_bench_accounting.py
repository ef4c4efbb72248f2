"""The bench's accounting helpers (CPU): screening keys, the count of
primitive quartets that pass the reference's screening (the roofline's FLOP
numerator), the FLOP convention, and the per-quartet DRAM traffic figure."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from librint_b200 import synthetic  # noqa: E402


def _data(cls, nq, seed=5):
    m, shls = synthetic.eri_sweep(cls, nq, seed=seed)
    return m.atm, m.bas, m.env, shls


def _cce_scalar(atm, bas, env, si, sj):
    """Screening keys of the primitive pairs of shells si, sj, one by one:
    mu R^2 - log_rr - log|c_i| - log|c_j| with log_rr = 1.7 - 1.5 log(a_i,min
    + a_j,min) + l_ij log(R + 1) (reference src/optimizer.rs:732-808)."""
    b = bas.reshape(-1, 8)
    a6 = atm.reshape(-1, 6)
    bi, bj = b[si], b[sj]
    ri = env[a6[bi[0], 1]:a6[bi[0], 1] + 3]
    rj = env[a6[bj[0], 1]:a6[bj[0], 1] + 3]
    rr = float(((ri - rj) ** 2).sum())
    lij = int(bi[1] + bj[1])
    log_rr = 1.7 - 1.5 * math.log(env[bi[5] + bi[2] - 1] + env[bj[5] + bj[2] - 1])
    if lij > 0:
        log_rr += lij * math.log(math.sqrt(rr) + 1.0)
    out = {}
    for jp in range(bj[2]):
        for ip in range(bi[2]):
            ai, aj = env[bi[5] + ip], env[bj[5] + jp]
            ci, cj = env[bi[6] + ip], env[bj[6] + jp]
            out[(ip, jp)] = (rr * ai * aj / (ai + aj) - log_rr - math.log(abs(ci))
                             - math.log(abs(cj)))
    return out


def test_pair_keys_match_scalar_restatement():
    atm, bas, env, shls = _data((2, 1, 1, 0), 24)
    keys = bench._pair_cce(bas, env, atm, shls[:, 0], shls[:, 1])
    b = bas.reshape(-1, 8)
    for q in range(shls.shape[0]):
        ref = _cce_scalar(atm, bas, env, shls[q, 0], shls[q, 1])
        ki, kj = b[shls[q, 0], 2], b[shls[q, 1], 2]
        row = keys[q].reshape(6, 6)
        for (ip, jp), v in ref.items():
            assert abs(row[ip, jp] - v) <= 1e-12 * max(1.0, abs(v))
        # absent primitives never pass
        assert np.isinf(row[ki:, :]).all() and np.isinf(row[:, kj:]).all()


def test_screened_count_matches_brute_force():
    cut = 60.0
    for cls in ((1, 1, 1, 1), (2, 2, 1, 0)):
        atm, bas, env, shls = _data(cls, 40)
        want = 0
        for q in range(shls.shape[0]):
            bra = _cce_scalar(atm, bas, env, shls[q, 0], shls[q, 1]).values()
            ket = _cce_scalar(atm, bas, env, shls[q, 2], shls[q, 3]).values()
            for kc in ket:
                if not kc <= cut:
                    continue
                want += sum(1 for bc in bra if bc + kc <= cut)
        assert bench.screened_prim_quartets(atm, bas, env, shls, cut) == want


def test_flop_convention_consistent():
    """class_flops with the unscreened primitive count equals
    class_flops_bytes' FLOPs, and screening can only lower it."""
    cls = (2, 1, 2, 1)
    atm, bas, env, shls = _data(cls, 32)
    f_all, nbytes = bench.class_flops_bytes(cls, bas, shls)
    k = bas.reshape(-1, 8)[:, 2][shls].astype(np.int64)
    assert bench.class_flops(cls, int(k.prod(axis=1).sum()), shls.shape[0]) == f_all
    passing = bench.screened_prim_quartets(atm, bas, env, shls)
    assert bench.class_flops(cls, passing, shls.shape[0]) <= f_all
    # bytes: 5 x 3 x 5 x 3 spherical doubles written per quartet plus pair data
    assert nbytes >= 8 * 225 * shls.shape[0]


def test_traffic_figure_close_to_algorithmic_bytes():
    """The measured (dd|dd) DRAM bytes per quartet are the 625 spherical
    output doubles plus pair data: within 10 % of the algorithmic bytes of the
    same workload."""
    cls = (2, 2, 2, 2)
    atm, bas, env, shls = _data(cls, 4096, seed=2)
    _, nbytes = bench.class_flops_bytes(cls, bas, shls)
    per_q = nbytes / shls.shape[0]
    assert 8 * 625 < per_q < 8 * 700
    assert abs(bench.NCU_TRAFFIC_PER_QUARTET[cls] / per_q - 1.0) < 0.10


def test_screening_profile_matches_the_screened_count():
    """The K^4-binned screening profile sums to screened_prim_quartets and to
    the unscreened primitive quartets, and puts each quartet in its bin."""
    for cls in [(0, 0, 0, 0), (2, 1, 1, 0), (2, 2, 2, 2)]:
        atm, bas, env, shls = _data(cls, 3000, seed=9)
        prof = bench.screening_profile(atm, bas, env, shls, chunk=1000)
        assert prof[:, 0].sum() == 3000
        k = bas.reshape(-1, 8)[:, 2][shls].astype(np.int64).prod(axis=1)
        assert prof[:, 1].sum() == k.sum()
        assert prof[:, 2].sum() == bench.screened_prim_quartets(atm, bas, env, shls)
        assert prof[0, 0] == np.count_nonzero(k == 1)
    data = [(c,) + _data(c, 500, seed=3) for c in [(1, 0, 0, 0), (2, 2, 1, 1)]]
    summ = bench.screening_summary(data, sample=400)
    assert set(summ["classes"]) == {"1000", "2211"}
    assert sum(b["quartets"] for b in summ["k4_bins"]) == 800
    assert 0.0 < summ["fraction_passed"] <= 1.0


def test_merged_sweep_layout():
    """The end-to-end leg's one-call layout: every quartet of the merged
    molecule names shells with the same angular momentum, primitives,
    exponents, coefficients and centres as in its own class; the merged
    arrays pass the library's host checks (on a machine without a GPU the
    call then stops at the first CUDA call, not at an input error), and the
    packed output length is the classes' lengths summed."""
    from librint_b200 import _bindings as B
    from librint_b200 import eri
    from librint_b200.basis import Molecule
    data = [(c,) + _data(c, 700, seed=4) for c in [(0, 0, 0, 0), (2, 1, 1, 0), (2, 2, 2, 2)]]
    offs, (na, nb, ne, no) = bench.merged_layout(data)
    nq = sum(d[4].shape[0] for d in data)
    atm = np.empty(6 * na, np.int32)
    bas = np.empty(8 * nb, np.int32)
    env = np.empty(ne)
    shl = np.empty(4 * nq, np.int32)
    bench.fill_merged(data, offs, atm, bas, env, shl)
    A, Bm, S = atm.reshape(-1, 6), bas.reshape(-1, 8), shl.reshape(-1, 4)
    q0 = 0
    for (cls, a, b, e, sh), (oa, ob, oe, oo) in zip(data, offs):
        a, b = a.reshape(-1, 6), b.reshape(-1, 8)
        for q in (0, 350, 699):
            for k in range(4):
                s_old, s_new = sh[q, k], S[q0 + q, k]
                bo, bn = b[s_old], Bm[s_new]
                assert bn[1] == bo[1] and bn[2] == bo[2]
                K = bo[2]
                np.testing.assert_array_equal(env[bn[5]:bn[5] + K], e[bo[5]:bo[5] + K])
                np.testing.assert_array_equal(env[bn[6]:bn[6] + K], e[bo[6]:bo[6] + K])
                pc_o, pc_n = a[bo[0], 1], A[bn[0], 1]
                np.testing.assert_array_equal(env[pc_n:pc_n + 3], e[pc_o:pc_o + 3])
        q0 += sh.shape[0]
    m = Molecule(atm, bas, env)
    assert eri.batch_len(m, S, 1) == no == sum(eri.batch_len(Molecule(d[1], d[2], d[3]), d[4], 1)
                                              for d in data)
    import torch
    if not torch.cuda.is_available():
        out = np.empty(no)
        rc = B.lib().lrb_int2e_batch(out.ctypes.data_as(B.P_d), 1, shl.ctypes.data_as(B.P_i), nq,
                                     atm.ctypes.data_as(B.P_i), na, bas.ctypes.data_as(B.P_i), nb,
                                     env.ctypes.data_as(B.P_d), ne)
        assert rc == -4, B.lib().lrb_last_error()
