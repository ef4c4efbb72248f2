"""Python front end of the batched ERI engine (host NumPy or device torch)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _bindings as B
from .basis import Molecule


def _arr(m: Molecule):
    return (np.ascontiguousarray(m.atm, dtype=np.int32), np.ascontiguousarray(m.bas, dtype=np.int32),
            np.ascontiguousarray(m.env, dtype=np.float64))


def batch_len(m: Molecule, shls, coord: int = 1) -> int:
    _, bas, _ = _arr(m)
    sh = np.ascontiguousarray(shls, dtype=np.int32)
    n = B.lib().lrb_int2e_batch_len(coord, sh.ctypes.data_as(B.P_i), sh.shape[0],
                                    bas.ctypes.data_as(B.P_i), bas.size // 8)
    if n < 0:
        raise B.LibrintError("bad quartet list")
    return n


def int2e_batch(m: Molecule, shls, coord: int = 1, out: np.ndarray | None = None) -> np.ndarray:
    """Packed libcint blocks of the quartets ``shls`` ((nq, 4) int32)."""
    atm, bas, env = _arr(m)
    sh = np.ascontiguousarray(shls, dtype=np.int32).reshape(-1, 4)
    n = batch_len(m, sh, coord)
    if out is None:
        out = np.empty(n)
    rc = B.lib().lrb_int2e_batch(out.ctypes.data_as(B.P_d), coord, sh.ctypes.data_as(B.P_i),
                                 sh.shape[0], atm.ctypes.data_as(B.P_i), atm.size // 6,
                                 bas.ctypes.data_as(B.P_i), bas.size // 8,
                                 env.ctypes.data_as(B.P_d), env.size)
    B.check(rc, "lrb_int2e_batch")
    return out


def int2e_batch_device(out, coord, shls, atm, bas, env, stream=None):
    """Device (torch.cuda) tensors in and out; queued on ``stream``."""
    import torch
    st = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = B.lib().lrb_int2e_batch_device(out.data_ptr(), coord, shls.data_ptr(), shls.numel() // 4,
                                        atm.data_ptr(), atm.numel() // 6, bas.data_ptr(),
                                        bas.numel() // 8, env.data_ptr(), env.numel(), st)
    B.check(rc, "lrb_int2e_batch_device")
    return out


def int2e(m: Molecule, coord: int = 0) -> np.ndarray:
    """Dense (n,n,n,n) tensor, reference integral2e layout (src/scf.rs:215)."""
    atm, bas, env = _arr(m)
    L = B.lib()
    ptr = L.int2e_c(atm.ctypes.data_as(B.P_i), atm.size, bas.ctypes.data_as(B.P_i), bas.size,
                    env.ctypes.data_as(B.P_d), env.size, coord)
    if not ptr:
        raise B.LibrintError("int2e_c failed: " + L.lrb_last_error().decode())
    n = m.nao(coord)
    out = np.ctypeslib.as_array(ptr, shape=(n ** 4,)).copy()
    L.free_c(ptr, n ** 4)
    return out.reshape(n, n, n, n)


def int2e_block(m: Molecule, shls, coord: int = 1, dims=None):
    """libcint per-quartet ABI (int2e_sph / int2e_cart), for drop-in checks."""
    atm, bas, env = _arr(m)
    b = bas.reshape(-1, 8)
    d = [((b[s, 1] + 1) * (b[s, 1] + 2) // 2 if coord == 0 else 2 * b[s, 1] + 1) * b[s, 3] for s in shls]
    out = np.zeros(int(np.prod(d)))
    sh = np.array(shls, dtype=np.int32)
    f = B.lib().int2e_cart if coord == 0 else B.lib().int2e_sph
    nz = f(out.ctypes.data_as(B.P_d), None, sh.ctypes.data_as(B.P_i), atm.ctypes.data_as(B.P_i),
           atm.size // 6, bas.ctypes.data_as(B.P_i), bas.size // 8, env.ctypes.data_as(B.P_d),
           None, None)
    return out.reshape(d[::-1]).transpose(3, 2, 1, 0), nz
