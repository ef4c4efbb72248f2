"""GPU test of lrb_int2e_batch_device_noalloc, the batched-ERI entry point for
callers that may not allocate device memory (for example inside a framework
whose caching allocator already holds the GPU's free memory).  It must give
the same integrals as lrb_int2e_batch_device, call after call, while taking
all scratch from its fixed static array: once warm, its calls change neither
the device's free memory nor the stream-ordered pool's reserved or used bytes.
This file sorts last so that a run stopping at the first failure has run every
other test before it."""
import ctypes

import numpy as np
import pytest

from librint_b200 import _bindings as B
from librint_b200 import eri, synthetic
from librint_b200.basis import Molecule
from tests.conftest import assert_eri_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LRB_ERR_INPUT = -1
MAX_QUARTETS = 65536


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _noalloc(out, coord, sh, atm, bas, env):
    st = torch.cuda.current_stream().cuda_stream
    return B.lib().lrb_int2e_batch_device_noalloc(out.data_ptr(), coord, sh.data_ptr(),
                                                  sh.numel() // 4, atm.data_ptr(), atm.numel() // 6,
                                                  bas.data_ptr(), bas.numel() // 8, env.data_ptr(),
                                                  env.numel(), ctypes.c_void_p(st))


class _DriverMemory:
    """Device free memory (cuMemGetInfo) and the default stream-ordered
    pool's reserved / used bytes (cuMemPoolGetAttribute), read through the
    CUDA driver on the calling thread's current context."""

    RESERVED_CURRENT, RESERVED_HIGH, USED_CURRENT, USED_HIGH = 5, 6, 7, 8

    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuCtxGetDevice(ctypes.byref(dev)) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def snapshot(self):
        free, total = ctypes.c_size_t(), ctypes.c_size_t()
        assert self.cu.cuMemGetInfo_v2(ctypes.byref(free), ctypes.byref(total)) == 0
        out = {"free": free.value}
        for name, attr in (("reserved", self.RESERVED_CURRENT), ("reserved_high", self.RESERVED_HIGH),
                           ("used", self.USED_CURRENT), ("used_high", self.USED_HIGH)):
            v = ctypes.c_uint64()
            assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
            out[name] = v.value
        return out


def _batches(golden):
    """A real molecule with shared shells and a high-momentum sweep class."""
    m = Molecule(golden["mol/h2o/def2svp/atm"], golden["mol/h2o/def2svp/bas"],
                 golden["mol/h2o/def2svp/env"])
    rng = np.random.default_rng(21)
    yield "h2o/def2svp", m, rng.integers(0, m.nbas, size=(4000, 4)).astype(np.int32)
    for cls in ((2, 2, 2, 1), (1, 0, 1, 0)):
        ms, sh = synthetic.eri_sweep(cls, 700, seed=23)
        yield "sweep%d%d%d%d" % cls, ms, sh


def test_noalloc_matches_batch_device_twice(golden):
    for name, m, shls in _batches(golden):
        atm, bas, env = _dev(m.atm, np.int32), _dev(m.bas, np.int32), _dev(m.env, np.float64)
        sh = _dev(shls, np.int32)
        for coord in (0, 1):
            n = eri.batch_len(m, shls, coord)
            ref = torch.empty(n, dtype=torch.float64, device="cuda")
            eri.int2e_batch_device(ref, coord, sh, atm, bas, env)
            for call in range(2):          # the second call reuses the shared scratch
                out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
                rc = _noalloc(out, coord, sh, atm, bas, env)
                assert rc == 0, B.lib().lrb_last_error().decode()
                torch.cuda.synchronize()
                assert_eri_close(out.cpu().numpy(), ref.cpu().numpy(),
                                 what=f"{name} coord {coord} call {call}")


def test_noalloc_allocates_no_device_memory(golden):
    """After a warm-up call (which places the static array and sets up the
    kernel table), further calls leave the device's free memory and the
    default pool's reserved / used bytes and their high-water marks as they
    were; every input and output is allocated before the first reading."""
    batches = []
    for name, m, shls in _batches(golden):
        d = dict(atm=_dev(m.atm, np.int32), bas=_dev(m.bas, np.int32), env=_dev(m.env, np.float64),
                 sh=_dev(shls, np.int32))
        d["out"] = torch.empty(eri.batch_len(m, shls, 1), dtype=torch.float64, device="cuda")
        batches.append(d)
    for d in batches:                      # warm-up
        assert _noalloc(d["out"], 1, d["sh"], d["atm"], d["bas"], d["env"]) == 0
    torch.cuda.synchronize()
    mem = _DriverMemory()
    before = mem.snapshot()
    for _ in range(3):
        for d in batches:
            rc = _noalloc(d["out"], 1, d["sh"], d["atm"], d["bas"], d["env"])
            assert rc == 0, B.lib().lrb_last_error().decode()
    torch.cuda.synchronize()
    after = mem.snapshot()
    assert after == before, (before, after)


def test_noalloc_rejects_batches_beyond_its_scratch():
    # too many quartets: rejected before any GPU work
    m, shls = synthetic.eri_sweep((0, 0, 0, 0), 8, seed=5)
    atm, bas, env = _dev(m.atm, np.int32), _dev(m.bas, np.int32), _dev(m.env, np.float64)
    big = np.zeros((MAX_QUARTETS + 1, 4), dtype=np.int32)
    out = torch.empty(MAX_QUARTETS + 1, dtype=torch.float64, device="cuda")
    assert _noalloc(out, 1, _dev(big, np.int32), atm, bas, env) == LRB_ERR_INPUT
    assert "split the batch" in B.lib().lrb_last_error().decode()
    # too many primitive pairs: (dd|dd) with up to 6 primitives per shell
    m, shls = synthetic.eri_sweep((2, 2, 2, 2), MAX_QUARTETS, seed=5)
    atm, bas, env = _dev(m.atm, np.int32), _dev(m.bas, np.int32), _dev(m.env, np.float64)
    out = torch.empty(eri.batch_len(m, shls, 1), dtype=torch.float64, device="cuda")
    assert _noalloc(out, 1, _dev(shls, np.int32), atm, bas, env) == LRB_ERR_INPUT
    assert "primitive pairs" in B.lib().lrb_last_error().decode()
    # and a batch that fits still works afterwards
    m, shls = synthetic.eri_sweep((1, 1, 0, 0), 300, seed=6)
    atm, bas, env = _dev(m.atm, np.int32), _dev(m.bas, np.int32), _dev(m.env, np.float64)
    sh = _dev(shls, np.int32)
    n = eri.batch_len(m, shls, 1)
    ref = torch.empty(n, dtype=torch.float64, device="cuda")
    eri.int2e_batch_device(ref, 1, sh, atm, bas, env)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    assert _noalloc(out, 1, sh, atm, bas, env) == 0, B.lib().lrb_last_error().decode()
    torch.cuda.synchronize()
    assert_eri_close(out.cpu().numpy(), ref.cpu().numpy(), what="after rejection")
