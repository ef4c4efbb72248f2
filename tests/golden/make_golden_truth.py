"""Golden one-electron Jacobians from the reference's own checks.

The reference's Rust checks (checks/overlap.rs, kinetic.rs, nuclear.rs)
store the Enzyme Jacobians d{S,T,V}/d env of H2 and H2O (STO-3G), over every
env entry (coordinates included), as text under checks/truth/.  This script
reads those text files and the molecules they belong to and stores them as a
small .npz next to this file; nothing is computed here.  Layout (from
checks/overlap.rs:96-175): J[k * m + l] = d O_k / d env[l], k = nu * n + mu,
m = len(env).

Run (needs the reference checkout, only in the development container):
    python tests/golden/make_golden_truth.py [/path/to/reference]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from librint_b200.basis import read_molecule  # noqa: E402

if len(sys.argv) < 2:
    sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
REF = sys.argv[1]


def main():
    out = {}
    for key in ("h2", "h2o"):
        m = read_molecule(os.path.join(REF, "molecules", key, "sto3g.txt"))
        out[f"truth/{key}/atm"], out[f"truth/{key}/bas"], out[f"truth/{key}/env"] = m.atm, m.bas, m.env
        n, L = m.nao(0), m.env.size
        # reverse mode for S and V; forward mode for T: the reverse-mode
        # kinetic truth of H2O disagrees with the forward-mode one (by up to
        # 0.48 in p-shell elements) and with central differences of the
        # reference's own T matrix, while the forward-mode one agrees (3.8e-9)
        for op, mode in (("dS", "rev"), ("dT", "for"), ("dV", "rev")):
            path = os.path.join(REF, "checks", "truth", key, f"sto3g_{op}_{mode}.txt")
            J = np.loadtxt(path)
            assert J.size == n * n * L, (key, op, J.size, n, L)
            out[f"truth/{key}/{op}"] = J.reshape(n * n, L)
        print(key, n, L, flush=True)
    np.savez_compressed(os.path.join(HERE, "reference_truth.npz"), **out)


if __name__ == "__main__":
    main()
