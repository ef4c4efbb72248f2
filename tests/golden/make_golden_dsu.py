"""Golden fixtures for dS_u (overlap Jacobian with respect to env[s1:s2]),
generated by calling the reference's shipped ``python/librint/librint.so``
through its exported ``dS_u`` entry point (src/p2c.rs:131,
src/dscf.rs:96-151), the same way make_golden.py calls the other entry
points.  The library is only called, never inspected.

Layout of the reference's result: element (nu * n + mu) * L + l is
d S[mu, nu] / d env[s1 + l], n cartesian AOs, L = s2 - s1.

Run (needs the reference checkout, only in the development container):
    python tests/golden/make_golden_dsu.py [/path/to/reference]
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from librint_b200 import synthetic  # noqa: E402
from librint_b200.basis import read_molecule  # noqa: E402
from make_golden import LIBC, P, _args, grad_len, mol_arrays  # noqa: E402

if len(sys.argv) < 2:
    sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
REF = sys.argv[1]


def main():
    lib = ctypes.CDLL(os.path.join(REF, "python", "librint", "librint.so"))
    a6 = (P(ctypes.c_int), ctypes.c_size_t, P(ctypes.c_int), ctypes.c_size_t,
          P(ctypes.c_double), ctypes.c_size_t)
    lib.dS_u.argtypes = a6
    lib.dS_u.restype = ctypes.c_void_p
    out = {}
    for key, m in (("h2", read_molecule(os.path.join(REF, "molecules/h2/sto3g.txt"))),
                   ("h2o", read_molecule(os.path.join(REF, "molecules/h2o/sto3g.txt"))),
                   ("water_like", synthetic.water_like())):
        n, L = m.nao(0), grad_len(m)
        ptr = lib.dS_u(*_args(m))
        a = np.ctypeslib.as_array(ctypes.cast(ptr, P(ctypes.c_double)), shape=(n * n * L,)).copy()
        LIBC.free(ptr)
        out.update(mol_arrays(f"dsu/{key}", m))
        out[f"dsu/{key}/dS_u"] = a
        print(key, n, L, float(np.abs(a).max()), flush=True)
    np.savez_compressed(os.path.join(HERE, "reference_dsu.npz"), **out)


if __name__ == "__main__":
    main()
