"""Fixture of the C3 energy test (tests/test_gpu_configs.py).

    python tests/golden/make_c3_energy.py <density.npz> [threads]

<density.npz> holds a converged FP64 RHF density of synthetic.c3_cluster()
(660 cartesian AOs) as written by the GPU SCF: ``P`` = the upper triangle
(row-major, numpy.triu_indices order) rounded to float32, ``n``, and ``E``
= the SCF energy.  The density is kept exactly as stored (float32 values,
symmetric); the oracle evaluates the energy functional at it through its
unique-quartet two-electron sum (about half an hour on 8 cores), and the
fixture tests/golden/c3_energy.npz records P, n, E_scf = E and E_oracle.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from librint_b200 import synthetic  # noqa: E402


def main():
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <density.npz> [threads]")
    f = np.load(sys.argv[1])
    threads = int(sys.argv[2]) if len(sys.argv) > 2 else 0
    n = int(f["n"])
    m = synthetic.c3_cluster()
    assert m.nao(0) == n
    P32 = f["P"].astype(np.float32)
    P = np.zeros((n, n))
    P[np.triu_indices(n)] = P32.astype(np.float64)
    P = P + np.triu(P, 1).T
    t0 = time.time()
    e = oracle.energy_sym(m, P, nthreads=threads)
    print(f"E_oracle = {e:.12f} ({time.time() - t0:.0f} s); E_scf = {float(f['E']):.12f}")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c3_energy.npz")
    np.savez_compressed(out, P=P32, n=n, E_scf=float(f["E"]), E_oracle=e)


if __name__ == "__main__":
    main()
