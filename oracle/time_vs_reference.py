"""Single-core speed of the oracle against the reference's shipped library.

The CPU baseline of bench.py is the oracle (a C++ restatement of the
reference's ERI path, OpenMP over quartets), because the reference is a Rust
crate that cannot be built here and its shipped ``python/librint/librint.so``
exists only in the reference checkout.  This script shows, on the host it
runs on, how fast that restatement is per core compared with the shipped
library on the same shell quartets: for every class of the ERI sweep it draws
8-shell molecules from the sweep's distribution (K = 1..6, exponents
log-uniform in [0.05, 5000], centres in a 10 A cube), times the reference's
``int2e_c`` (all nbas^4 quartets of the molecule, spherical, one core; the
reference builds libcint's optimizer once per call, src/scf.rs:236-250), and
times the oracle's dense tensor of the same molecule (orc_int2e_tensor: the
same nbas^4 quartets, pair data built once per call) on one thread.  The
library is only called through its exported C entry point
(src/p2c.rs:109), as python/librint/_bindings.py does.

Run (needs the reference checkout, only in the development container):
    python oracle/time_vs_reference.py <path of the reference checkout> [molecules per class]
"""
from __future__ import annotations

import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from librint_b200 import synthetic  # noqa: E402

P = ctypes.POINTER


def load_ref(ref):
    lib = ctypes.CDLL(os.path.join(ref, "python", "librint", "librint.so"))
    lib.int2e_c.argtypes = (P(ctypes.c_int), ctypes.c_size_t, P(ctypes.c_int), ctypes.c_size_t,
                            P(ctypes.c_double), ctypes.c_size_t, ctypes.c_int)
    lib.int2e_c.restype = ctypes.c_void_p
    return lib


def main():
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout> "
                 f"[molecules per class]")
    ref = load_ref(sys.argv[1])
    per_class = int(sys.argv[2]) if len(sys.argv) > 2 else 4
    libc = ctypes.CDLL("libc.so.6")
    libc.free.argtypes = (ctypes.c_void_p,)
    rows = []
    tr_all = to_all = 0.0
    nq_all = 0
    for cls in synthetic.canonical_classes(2):
        tr = to = 0.0
        nq = 0
        for r in range(per_class):
            m, _ = synthetic.eri_sweep(cls, 2, seed=4000 + r)
            atm = np.ascontiguousarray(m.atm, dtype=np.int32)
            bas = np.ascontiguousarray(m.bas, dtype=np.int32)
            env = np.ascontiguousarray(m.env, dtype=np.float64)
            nb = bas.size // 8
            t0 = time.perf_counter()
            ptr = ref.int2e_c(atm.ctypes.data_as(P(ctypes.c_int)), atm.size,
                              bas.ctypes.data_as(P(ctypes.c_int)), bas.size,
                              env.ctypes.data_as(P(ctypes.c_double)), env.size, 1)
            tr += time.perf_counter() - t0
            if not ptr:
                sys.exit(f"reference int2e_c failed for class {cls}")
            libc.free(ptr)
            t0 = time.perf_counter()
            oracle.int2e_tensor(m, 1, nthreads=1)
            to += time.perf_counter() - t0
            nq += nb ** 4
        rows.append((cls, nq, nq / tr, nq / to))
        tr_all += tr
        to_all += to
        nq_all += nq
    print("class       quartets   reference q/s   oracle q/s (1 thread)   oracle / reference")
    for cls, nq, r, o in rows:
        print("(%d%d|%d%d)  %9d  %14.0f  %22.0f  %8.2f" % (cls + (nq, r, o, o / r)))
    print("all classes %9d  %14.0f  %22.0f  %8.2f" % (nq_all, nq_all / tr_all, nq_all / to_all,
                                                      tr_all / to_all))


if __name__ == "__main__":
    main()
