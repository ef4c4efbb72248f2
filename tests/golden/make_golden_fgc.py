"""Golden fixtures for f shells and generally contracted shells, from the
reference's own shipped library (called through ctypes as make_golden.py
does; the library is never inspected).

    python tests/golden/make_golden_fgc.py <path of the reference checkout>

Writes tests/golden/reference_fgc.npz:
* ``f/<class>/<q>/...``: for every canonical class with an f shell, three
  compact 4-shell molecules (centres within +-1.5 Bohr, 1..3 primitives,
  exponents log-uniform in [0.15, 30]) and their (ij|kl) blocks from the
  reference's int2e_c, cartesian and spherical;
* ``gc/...``: a water-like molecule with generally contracted shells (O s
  and p with 2 and 3 contractions, H s with 2): int1e, 30,000 sampled
  elements of the cartesian and spherical int2e_c tensors, and the
  reference's SCF energy and density (conv 1e-10);
* ``fpol/...``: the same geometry with O d and f and H p polarisation
  shells: int1e, sampled int2e_c, SCF energy and density;
* ``rs/<mol>/<omega>/...``: range-separated int2e_c (env[8] = omega) of the
  water-like molecule (full tensors) and of h2o/def2svp (30,000 sampled
  elements): long range (omega = 0.3) everywhere, short range (omega =
  -0.3) only for elements of shell quartets of Rys order <= 3.  For orders
  >= 4 the shipped library's short-range nodes are wrong (a (dd|dd) element
  of h2o/def2svp comes out 5.912 where the 40-digit value is 3.939) and at
  omega = -2 its node solver aborts the process, so those are pinned against
  the 40-digit evaluation instead (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from make_golden import _args, _take, load_ref, mol_arrays  # noqa: E402
from librint_b200 import synthetic  # noqa: E402
from librint_b200.basis import BOHR, Builder, Molecule  # noqa: E402


def f_classes():
    return [c for c in synthetic.canonical_classes(3) if max(c) == 3]


def compact_quartet(rng, cls):
    b = Builder()
    for l in cls:
        at = b.add_atom(1, rng.uniform(-1.5, 1.5, 3))
        k = int(rng.integers(1, 4))
        e = np.sort(np.exp(rng.uniform(math.log(0.15), math.log(30.0), k)))[::-1]
        b.add_shell(at, l, e, rng.uniform(0.2, 1.0, k))
    return b.build("quartet")


def rys_order_of_elements(m, coord):
    """Rys order (li+lj+lk+ll)/2 + 1 of the shell quartet of every element of
    the n^4 tensor (flat)."""
    b = m.bas.reshape(-1, 8)
    l_ao = np.concatenate([[l] * (((l + 1) * (l + 2) // 2 if coord == 0 else 2 * l + 1) * nc)
                           for l, nc in zip(b[:, 1], b[:, 3])])
    L = (l_ao[:, None, None, None] + l_ao[None, :, None, None] + l_ao[None, None, :, None] +
         l_ao[None, None, None, :])
    return (L // 2 + 1).ravel()


def water_geometry(b):
    o = b.add_atom(8, np.array([0.0, 0.0, 0.117]) / BOHR)
    h1 = b.add_atom(1, np.array([0.0, 0.757, -0.467]) / BOHR)
    h2 = b.add_atom(1, np.array([0.0, -0.757, -0.467]) / BOHR)
    return o, (h1, h2)


def gc_water(rng):
    b = Builder()
    o, hs = water_geometry(b)
    e = np.sort(np.exp(rng.uniform(math.log(0.2), math.log(150.0), 5)))[::-1]
    b.add_shell_gc(o, 0, e, [rng.uniform(0.2, 1, 5), rng.uniform(-1, 1, 5)])
    b.add_shell_gc(o, 1, e[1:], [rng.uniform(0.2, 1, 4), rng.uniform(0.2, 1, 4),
                                 rng.uniform(-1, 1, 4)])
    b.add_shell(o, 2, [0.8], [1.0])
    for h in hs:
        b.add_shell_gc(h, 0, [5.0, 0.8, 0.2], [[0.3, 0.6, 0.4], [0.1, -0.5, 1.0]])
    return b.build("gc_water")


def fpol_water(rng):
    b = Builder()
    o, hs = water_geometry(b)
    e = np.sort(np.exp(rng.uniform(math.log(0.2), math.log(150.0), 4)))[::-1]
    b.add_shell(o, 0, e, rng.uniform(0.2, 1, 4))
    b.add_shell(o, 0, [0.35], [1.0])
    b.add_shell(o, 1, e[:3], rng.uniform(0.2, 1, 3))
    b.add_shell(o, 2, [1.1, 0.4], [0.6, 0.5])
    b.add_shell(o, 3, [0.9], [1.0])
    for h in hs:
        b.add_shell(h, 0, [8.0, 1.2, 0.25], [0.2, 0.5, 0.6])
        b.add_shell(h, 1, [0.7], [1.0])
    return b.build("fpol_water")


def molecule_set(lib, rng, key, m, out):
    out.update(mol_arrays(key, m))
    for coord in (0, 1):
        n = m.nao(coord)
        for typec in (0, 1, 2):
            out[f"{key}/int1e_{coord}{typec}"] = _take(lib.int1e_c(*_args(m), coord, typec),
                                                       n * n).reshape(n, n)
        t = _take(lib.int2e_c(*_args(m), coord), n ** 4)
        idx = np.sort(rng.choice(n ** 4, size=30000, replace=False))
        out[f"{key}/int2e_{coord}_idx"] = idx
        out[f"{key}/int2e_{coord}_val"] = t[idx]
    out[f"{key}/scf"] = lib.scf_c(*_args(m), m.nelec, 2000, 1e-10)
    n0 = m.nao(0)
    out[f"{key}/scf_P"] = _take(lib.density_c(*_args(m), m.nelec, 2000, 1e-10),
                                n0 * n0).reshape(n0, n0)
    print(key, "nao", n0, "E", out[f"{key}/scf"], flush=True)


def main():
    lib = load_ref()
    rng = np.random.default_rng(20261204)
    out = {}
    for cls in f_classes():
        for q in range(3):
            m = compact_quartet(rng, cls)
            key = "f/%d%d%d%d/%d" % (cls + (q,))
            out.update(mol_arrays(key, m))
            for coord, name in ((0, "cart"), (1, "sph")):
                d = [((l + 1) * (l + 2) // 2 if coord == 0 else 2 * l + 1) for l in cls]
                n = sum(d)
                t = _take(lib.int2e_c(*_args(m), coord), n ** 4).reshape(n, n, n, n)
                o = np.cumsum([0] + d)
                out[f"{key}/{name}"] = t[o[0]:o[1], o[1]:o[2], o[2]:o[3], o[3]:o[4]].copy()
        print("class", cls, flush=True)
    molecule_set(lib, rng, "gc", gc_water(rng), out)
    molecule_set(lib, rng, "fpol", fpol_water(rng), out)
    g = np.load(os.path.join(HERE, "reference_golden.npz"))
    svp = Molecule(g["mol/h2o/def2svp/atm"], g["mol/h2o/def2svp/bas"], g["mol/h2o/def2svp/env"], 10)
    for name, m in (("water_like", synthetic.water_like()), ("h2o_def2svp", svp)):
        for omega in (0.3, -0.3):
            env = m.env.copy()
            env[8] = omega
            mo = Molecule(m.atm, m.bas, env, m.nelec)
            key = f"rs/{name}/{omega:+.1f}"
            out.update(mol_arrays(key, mo))
            for coord in (0, 1):
                n = mo.nao(coord)
                t = _take(lib.int2e_c(*_args(mo), coord), n ** 4)
                keep = np.arange(n ** 4)
                if omega < 0:
                    keep = keep[rys_order_of_elements(mo, coord)[keep] <= 3]
                if keep.size > 30000:
                    keep = np.sort(rng.choice(keep, size=30000, replace=False))
                out[f"{key}/int2e_{coord}_idx"] = keep
                out[f"{key}/int2e_{coord}_val"] = t[keep]
            print(key, flush=True)
    path = os.path.join(HERE, "reference_fgc.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
