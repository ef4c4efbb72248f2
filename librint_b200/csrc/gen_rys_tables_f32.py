"""Generate rys_tables_f32.h, the single-precision Rys tables of the FP32
Fock kernels, from the double-precision tables in rys_tables.h.

Each segment polynomial of rys_tables.h (degree 18 in the local variable
t in [-1, 1]) is economised: converted to the Chebyshev basis, truncated to
degree DEG32 and converted back to monomial coefficients, which are then
rounded to float (Lanczos' Chebyshev economisation; the truncation error is
bounded by the sum of the dropped Chebyshev coefficients).  Only nroots up to
NMAX32 are written: the FP32 kernels cover classes up to (dd|dd), 5 roots.
The large-x limit is shared with the FP64 tables (RYS_LARGEX_R/W, rounded to
float at use).

Every function is validated on a dense grid of each segment against the
double-precision polynomial with the float coefficients evaluated in float
by Horner's rule; the script refuses to write a table whose worst relative
error exceeds TOL32.

Run:  python librint_b200/csrc/gen_rys_tables_f32.py   (writes rys_tables_f32.h)
"""
import os
import re
import sys

import numpy as np
from numpy.polynomial import chebyshev as cheb
from numpy.polynomial import polynomial as poly

HERE = os.path.dirname(os.path.abspath(__file__))
NMAX32 = 5
DEG32 = 10
TOL32 = 1.0e-6
NGRID = 401


def read_fp64_tables(path):
    """(deg, ncoef, nseg[], offset[], coefficients) of rys_tables.h."""
    src = open(path).read()
    deg = int(re.search(r"#define RYS_DEG (\d+)", src).group(1))
    ncoef = int(re.search(r"#define RYS_NCOEF (\d+)", src).group(1))
    nseg = [int(v) for v in re.search(r"RYS_TAB_NSEG\[[^]]*\] = \{([^}]*)\}", src).group(1).split(",")]
    off = [int(v) for v in re.search(r"RYS_TAB_OFFSET\[[^]]*\] = \{([^}]*)\}", src).group(1).split(",")]
    body = re.search(r"RYS_TAB\[(\d+)\] = \{([^}]*)\}", src)
    tab = np.array([float(v) for v in body.group(2).split(",") if v.strip()])
    assert len(tab) == int(body.group(1)) == off[-1]
    return deg, ncoef, nseg, off, tab


def horner_f32(c32, t32):
    r = np.full_like(t32, c32[-1])
    for k in range(len(c32) - 2, -1, -1):
        r = (r * t32 + c32[k]).astype(np.float32)
    return r


def economise(c):
    """Degree-DEG32 float coefficients of the monomial series c on [-1, 1]."""
    ch = cheb.poly2cheb(c)
    return cheb.cheb2poly(ch[:DEG32 + 1]).astype(np.float32)


def main():
    deg, ncoef, nseg, off, tab = read_fp64_tables(os.path.join(HERE, "rys_tables.h"))
    t = np.linspace(-1.0, 1.0, NGRID)
    t32 = t.astype(np.float32)
    out, offs, worst = [], [0, 0], []
    for n in range(1, NMAX32 + 1):
        w = 0.0
        for s in range(nseg[n]):
            for f in range(2 * n):
                b = off[n] + (s * 2 * n + f) * ncoef
                c = tab[b:b + ncoef]
                c32 = economise(c)
                exact = poly.polyval(t, c)
                got = horner_f32(c32, t32).astype(np.float64)
                w = max(w, float(np.max(np.abs(got - exact) / np.abs(exact))))
                out.extend(c32.tolist())
        if w > TOL32:
            sys.exit(f"nroots={n}: worst relative error {w:.2e} exceeds {TOL32:.0e}")
        worst.append(w)
        offs.append(len(out))
    lines = ["// Generated by gen_rys_tables_f32.py from rys_tables.h -- do not edit.",
             "// Single-precision Rys nodes and weights for the FP32 Fock kernels: the",
             f"// segment polynomials of rys_tables.h economised to degree {DEG32} (Chebyshev",
             "// truncation), float coefficients, same layout and local variable.",
             "// Worst relative error against the FP64 polynomials, float Horner:"]
    for n, w in enumerate(worst, 1):
        lines.append(f"// nroots={n}: {w:.2e}")
    lines += ["#pragma once",
              "#ifndef RYS_TAB_QUAL",
              "#define RYS_TAB_QUAL",
              "#endif",
              f"#define RYS32_NMAX {NMAX32}",
              f"#define RYS32_DEG {DEG32}",
              f"#define RYS32_NCOEF {DEG32 + 1}",
              "static constexpr int RYS32_TAB_OFFSET[RYS32_NMAX + 2] = {" +
              ", ".join(str(v) for v in offs) + "};",
              "#ifndef RYS_OMIT_TAB",
              f"RYS_TAB_QUAL static const float RYS32_TAB[{len(out)}] = {{"]
    for i in range(0, len(out), DEG32 + 1):
        lines.append("  " + ", ".join(f"{v!r}f" if "e" in repr(v) or "." in repr(v) else f"{v!r}.0f"
                                      for v in (float(np.float32(x)) for x in out[i:i + DEG32 + 1])) + ",")
    lines += ["};", "#endif"]
    with open(os.path.join(HERE, "rys_tables_f32.h"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    print("worst relative errors:", " ".join(f"{w:.2e}" for w in worst))


if __name__ == "__main__":
    main()
