"""GPU parity of the batched ERI engine, through the C ABI, against the CPU
oracle and the reference goldens (tolerance of tests/conftest.py)."""
import numpy as np
import pytest

import oracle
from librint_b200 import eri, synthetic
from librint_b200 import _bindings as B
from librint_b200.basis import Molecule
from tests.conftest import assert_eri_close, assert_eri_close_or_exact

pytestmark = pytest.mark.gpu

CLASSES = synthetic.canonical_classes(2)


def _blocks(m, shls, coord):
    """Oracle blocks for a quartet list, unpacked."""
    packed = oracle.int2e_batch(m, shls, coord)
    return packed


@pytest.mark.parametrize("cls", CLASSES)
def test_class_samples_vs_reference_golden(golden, cls):
    key = "cls/%d%d%d%d" % cls
    env = golden[key + "/env"]
    for q in range(golden[key + "/atm"].shape[0]):
        m = Molecule(golden[key + "/atm"][q].ravel(), golden[key + "/bas"][q].ravel(), env)
        for coord, nm in ((0, "cart"), (1, "sph")):
            got = eri.int2e_batch(m, [[0, 1, 2, 3]], coord)
            ref = golden[f"{key}/{nm}"][q]
            assert_eri_close(got, ref.transpose(3, 2, 1, 0).ravel(), what=f"{key} q{q} {nm}")


@pytest.mark.parametrize("coord", [0, 1])
def test_sweep_batch_vs_oracle(coord):
    """All 21 classes, 400 random quartets each, in one mixed batch."""
    for cls in CLASSES:
        m, shls = synthetic.eri_sweep(cls, 400, seed=11)
        got = eri.int2e_batch(m, shls, coord)
        ref = oracle.int2e_batch(m, shls, coord)
        assert_eri_close_or_exact(got, ref, m, shls, coord, lambda sh: eri.int2e_batch(m, sh, 0),
                                  what=f"class {cls} coord {coord}")


def test_permuted_shell_orders_vs_oracle():
    """Non-canonical quartet orders are canonicalised and written back in the
    requested layout."""
    rng = np.random.default_rng(5)
    for cls in [(2, 1, 1, 0), (2, 2, 2, 0), (1, 0, 1, 1), (2, 0, 2, 1)]:
        m, shls = synthetic.eri_sweep(cls, 60, seed=12)
        perms = [rng.permutation(4) for _ in range(shls.shape[0])]
        sh = np.array([s[p] for s, p in zip(shls, perms)], dtype=np.int32)
        for coord in (0, 1):
            assert_eri_close(eri.int2e_batch(m, sh, coord), oracle.int2e_batch(m, sh, coord),
                             what=f"perm {cls} {coord}")


def test_mixed_molecule_batch(golden):
    """Quartets of a real molecule (shared shells) in one batch."""
    m = Molecule(golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
                 golden["mol/h2o/def2svp/env"])
    rng = np.random.default_rng(3)
    sh = rng.integers(0, m.nbas, size=(3000, 4)).astype(np.int32)
    for coord in (0, 1):
        assert_eri_close(eri.int2e_batch(m, sh, coord), oracle.int2e_batch(m, sh, coord))


@pytest.mark.parametrize("name", ["h2o/sto3g", "ch4/sto3g", "lih/sto3g"])
def test_int2e_c_dense_vs_golden(golden, name):
    key = "mol/" + name
    m = Molecule(golden[key + "/atm"], golden[key + "/bas"], golden[key + "/env"])
    for coord in (0, 1):
        assert_eri_close(eri.int2e(m, coord), golden[f"{key}/int2e_{coord}"], what=name)


def test_int2e_c_subsample_def2svp(golden):
    key = "mol/h2o/def2svp"
    m = Molecule(golden[key + "/atm"], golden[key + "/bas"], golden[key + "/env"])
    for coord in (0, 1):
        t = eri.int2e(m, coord).ravel()
        assert_eri_close(t[golden[f"{key}/int2e_{coord}_idx"]], golden[f"{key}/int2e_{coord}_val"])


def test_libcint_per_quartet_abi(golden):
    m = synthetic.water_like()
    for shls in ([0, 1, 2, 3], [2, 2, 2, 2], [4, 2, 0, 2]):
        for coord in (0, 1):
            got, nz = eri.int2e_block(m, shls, coord)
            ref, _ = oracle.int2e_block(m, shls, coord)
            assert nz == 1
            assert_eri_close(got, ref)


def test_errors_are_reported_not_fatal():
    m, shls = synthetic.eri_sweep((1, 0, 0, 0), 4, seed=1)
    # empty batch is a no-op
    assert eri.int2e_batch(m, np.zeros((0, 4), np.int32)).size == 0
    # shell index out of range
    bad = shls.copy()
    bad[0, 0] = m.nbas + 7
    with pytest.raises(B.LibrintError):
        eri.int2e_batch(m, bad)
    # g shell: no kernel (l <= 3)
    m2 = Molecule(m.atm.copy(), m.bas.copy(), m.env.copy())
    m2.bas.reshape(-1, 8)[0, 1] = 4
    with pytest.raises(B.LibrintError):
        eri.int2e_batch(m2, shls[:1], 0)
    # more than 31 primitives in a shell
    m3 = Molecule(m.atm.copy(), m.bas.copy(), np.concatenate([m.env, np.ones(80)]))
    b3 = m3.bas.reshape(-1, 8)
    b3[0, 2] = 40
    b3[0, 5] = m.env.size
    b3[0, 6] = m.env.size + 40
    with pytest.raises(B.LibrintError):
        eri.int2e_batch(m3, shls[:1], 0)
    # the library still works afterwards
    assert_eri_close(eri.int2e_batch(m, shls), oracle.int2e_batch(m, shls, 1))


@pytest.mark.skipif(__import__("torch").cuda.device_count() < 2, reason="needs two GPUs")
def test_second_device_same_results():
    """Kernel tables, cart->sph coefficients and shared-memory limits are set
    up per device: spherical (dd|dd) blocks (> 48 KB of shared memory) and a
    Fock build on device 1 equal those of device 0 in the same process."""
    import torch
    from librint_b200 import scf
    m, shls = synthetic.eri_sweep((2, 2, 2, 2), 64, seed=5)
    mw = synthetic.water_like()
    P = np.eye(mw.nao(0))
    out = []
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        ctx = scf.MolContext(mw)
        out.append((eri.int2e_batch(m, shls, 1), ctx.fock_G(P, 0.0)))
        ctx.close()
    torch.cuda.set_device(0)
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-13, atol=1e-14)


def _pinned_batch(m, sh, coord):
    """lrb_int2e_batch into a page-locked output buffer (the copy-out of
    every chunk then runs on its own stream while later chunks compute)."""
    import ctypes
    import torch
    L = B.lib()
    n = eri.batch_len(m, sh, coord)
    out = torch.empty(n, dtype=torch.float64).pin_memory()
    rc = L.lrb_int2e_batch(ctypes.cast(out.data_ptr(), B.P_d), coord, sh.ctypes.data_as(B.P_i),
                           sh.shape[0], m.atm.ctypes.data_as(B.P_i), m.atm.size // 6,
                           m.bas.ctypes.data_as(B.P_i), m.bas.size // 8,
                           m.env.ctypes.data_as(B.P_d), m.env.size)
    B.check(rc, "lrb_int2e_batch")
    return out.numpy().copy()


def _sliced(m, sh, coord, step):
    return np.concatenate([eri.int2e_batch(m, np.ascontiguousarray(sh[i:i + step]), coord)
                           for i in range(0, sh.shape[0], step)])


def test_multichunk_batch_shared_molecule(golden):
    """600,000 quartets of one molecule (shared shells: the molecule goes up
    once, 3 chunks of <= 262,144 quartets pass through both device slots)
    equal the same quartets computed in single-chunk calls, bit for bit, with
    pageable and page-locked output; the first quartets match the oracle."""
    m = Molecule(golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
                 golden["mol/h2o/def2svp/env"])
    rng = np.random.default_rng(8)
    sh = rng.integers(0, m.nbas, size=(600_000, 4)).astype(np.int32)
    for coord in (0, 1):
        ref = _sliced(m, sh, coord, 100_000)
        np.testing.assert_array_equal(eri.int2e_batch(m, sh, coord), ref)
        np.testing.assert_array_equal(_pinned_batch(m, sh, coord), ref)
        head = np.ascontiguousarray(sh[:2000])
        assert_eri_close(ref[:eri.batch_len(m, head, coord)], oracle.int2e_batch(m, head, coord))


def test_multichunk_batch_streamed_molecule():
    """160,000 (dd|dd) quartets with their own shells (the sweep layout: each
    chunk uploads its own part of the molecule) in 3 output-bounded chunks
    equal single-chunk calls of 40,000 quartets, bit for bit, with pageable
    and page-locked output."""
    m, sh = synthetic.eri_sweep((2, 2, 2, 2), 160_000, seed=9)
    ref = _sliced(m, sh, 1, 40_000)
    np.testing.assert_array_equal(eri.int2e_batch(m, sh, 1), ref)
    np.testing.assert_array_equal(_pinned_batch(m, sh, 1), ref)
    head = np.ascontiguousarray(sh[:200])
    assert_eri_close_or_exact(ref[:eri.batch_len(m, head, 1)], oracle.int2e_batch(m, head, 1), m,
                              head, 1, lambda q: eri.int2e_batch(m, q, 0), what="streamed (dd|dd)")
