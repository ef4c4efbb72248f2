"""ctypes bindings of librint_b200/_lib/librint_b200.so.

Mirrors the reference's python/librint/_bindings.py (same p2c.rs entry points
and argument types, LIBRINT_SO environment override), plus this library's
own batched / device entry points.  Loading fails loudly: there is no CPU
fallback for any compute path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.environ.get("LIBRINT_SO", os.path.join(HERE, "_lib", "librint_b200.so"))

c_int, c_ll, c_sz, c_d, c_vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p
P_i = ctypes.POINTER(ctypes.c_int)
P_d = ctypes.POINTER(ctypes.c_double)

_lib = None


class LibrintError(RuntimeError):
    pass


# status codes (include/librint_b200.h)
LRB_OK, LRB_ERR_INPUT, LRB_ERR_UNSUPPORTED, LRB_ERR_ALLOC = 0, -1, -2, -3
LRB_ERR_CUDA, LRB_ERR_SCF, LRB_ERR_TIMEOUT = -4, -5, -6


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO_PATH):
        raise LibrintError(f"librint_b200 CUDA library not found at {SO_PATH}; "
                           "build it with `python -m librint_b200.build`")
    L = ctypes.CDLL(SO_PATH)
    L.lrb_last_error.restype = ctypes.c_char_p
    L.lrb_last_error.argtypes = ()
    L.lrb_int2e_batch_len.restype = c_ll
    L.lrb_int2e_batch_len.argtypes = (c_int, P_i, c_ll, P_i, c_int)
    L.lrb_int2e_batch.restype = c_int
    L.lrb_int2e_batch.argtypes = (P_d, c_int, P_i, c_ll, P_i, c_int, P_i, c_int, P_d, c_ll)
    L.lrb_int2e_batch_device.restype = c_int
    L.lrb_int2e_batch_device.argtypes = (c_vp, c_int, c_vp, c_ll, c_vp, c_int, c_vp, c_int, c_vp,
                                         c_ll, c_vp)
    for f in ("int2e_sph", "int2e_cart"):
        getattr(L, f).restype = c_int
        getattr(L, f).argtypes = (P_d, P_i, P_i, P_i, c_int, P_i, c_int, P_d, c_vp, P_d)
    L.int2e_optimizer.restype = None
    L.int2e_optimizer.argtypes = (ctypes.POINTER(c_vp), P_i, c_int, P_i, c_int, P_d)
    L.CINTdel_optimizer.restype = None
    L.CINTdel_optimizer.argtypes = (ctypes.POINTER(c_vp),)
    # librint p2c.rs ABI
    L.free_c.restype = None
    L.free_c.argtypes = (P_d, c_sz)
    L.int2e_c.restype = P_d
    L.int2e_c.argtypes = (P_i, c_sz, P_i, c_sz, P_d, c_sz, c_int)
    _optional(L)
    _lib = L
    return L


class ScfOptions(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("conv", ctypes.c_double), ("guess", ctypes.c_int),
                ("diis", ctypes.c_int), ("tau", ctypes.c_double), ("mixed", ctypes.c_int),
                ("fp32_until", ctypes.c_double), ("tau32", ctypes.c_double),
                ("rebuild_every", ctypes.c_int), ("tau_fp32", ctypes.c_double),
                ("tau_prim", ctypes.c_double)]


class ScfResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("e_nuc", ctypes.c_double), ("delta", ctypes.c_double),
                ("fock_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
                ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("quartets", ctypes.c_longlong), ("fp32_quartets", ctypes.c_longlong)]


def _optional(L):
    """Entry points added as the library grows; declared when present."""
    sigs = {
        "lrb_profile_enable": (None, (c_int,)),
        "lrb_profile_read": (c_int, (P_d, c_int)),
        "lrb_launch_count": (c_ll, ()),
        "lrb_fock_class_counts": (c_int, (ctypes.POINTER(c_ll), ctypes.POINTER(c_ll), c_int)),
        "lrb_fock_lane_min": (c_int, (c_int,)),
        "lrb_fp64_peak_probe": (c_d, (c_int,)),
        "lrb_mol_create": (c_int, (ctypes.POINTER(c_vp), P_i, c_int, P_i, c_int, P_d, c_ll)),
        "lrb_mol_destroy": (None, (c_vp,)),
        "lrb_mol_nao": (c_int, (c_vp,)),
        "lrb_mol_set_tau_prim": (c_int, (c_vp, c_d)),
        "lrb_fock_G": (c_int, (c_vp, P_d, P_d, c_d, ctypes.POINTER(c_ll))),
        "lrb_fock_G_device": (c_int, (c_vp, c_vp, c_vp, c_d, c_vp)),
        "lrb_fock_G_part": (c_int, (c_vp, P_d, P_d, c_d, c_int, c_int, ctypes.POINTER(c_ll))),
        "lrb_fock_G_part_device": (c_int, (c_vp, c_vp, c_vp, c_d, c_int, c_int,
                                           ctypes.POINTER(c_ll), c_vp)),
        "lrb_fock_G_prec": (c_int, (c_vp, P_d, P_d, c_d, c_int, c_d, ctypes.POINTER(c_ll),
                                    ctypes.POINTER(c_ll))),
        "lrb_scf": (c_int, (c_vp, c_ll, ctypes.POINTER(ScfOptions), ctypes.POINTER(ScfResult),
                            P_d, P_d)),
        "lrb_energy": (c_int, (c_vp, P_d, c_d, P_d)),
        "lrb_int1e": (c_int, (c_vp, c_int, c_int, P_d)),
        "int1e_c": (P_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz, c_int, c_int)),
        "density_c": (P_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz, c_sz, c_int, c_d)),
        "energy_c": (c_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz, P_d, c_sz)),
        "scf_c": (c_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz, c_sz, c_int, c_d)),
        "lrb_grad_len": (c_int, (c_vp,)),
        "lrb_grad": (c_int, (c_vp, P_d, c_d, c_d, c_d, c_d, P_d)),
        "lrb_grad_nuc": (c_int, (c_vp, P_d, c_d, P_d)),
        "lrb_int1e_jacobian": (c_int, (c_vp, c_int, P_d)),
        "lrb_int2e_batch_device_noalloc": (c_int, (c_vp, c_int, c_vp, c_ll, c_vp, c_int, c_vp,
                                                   c_int, c_vp, c_ll, c_vp)),
        "lrb_mlp_forward": (c_int, (c_vp, c_int, c_int, c_vp, c_vp, c_int, c_int, c_vp, c_vp,
                                    c_vp)),
        "lrb_mlp_backward": (c_int, (c_vp, c_int, c_int, c_vp, c_int, c_int, c_vp, c_vp, c_vp,
                                     c_vp, c_vp, c_vp, c_vp)),
        "lrb_mse": (c_int, (c_vp, c_vp, c_vp, c_ll, ctypes.c_float, c_vp, c_vp, c_vp)),
        "lrb_adam": (c_int, (c_vp, c_vp, c_vp, c_vp, c_ll, ctypes.c_float, ctypes.c_float,
                             ctypes.c_float, ctypes.c_float, c_int, c_vp)),
    }
    sigs["dS_u"] = (P_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz))
    for name in ("grad_c", "dS_c", "dHcore_c", "dR_c", "danalytical_c", "denergy_c"):
        sigs[name] = (P_d, (P_i, c_sz, P_i, c_sz, P_d, c_sz, P_d, c_sz))
    for name, (res, args) in list(sigs.items()):
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args


def check(rc: int, what: str = "librint_b200"):
    if rc != 0:
        msg = lib().lrb_last_error().decode()
        raise LibrintError(f"{what} failed ({rc}): {msg}")
