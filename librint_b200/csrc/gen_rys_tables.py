"""Generate the Rys quadrature tables used by the ERI kernels and the oracle.

Rys quadrature for a primitive quartet needs, for nroots = n and argument
x = a0 * |P - Q|^2, the n-point Gauss rule of the weight exp(-x t^2) on
t in [0, 1].  The librint ABI (and libcint before it) passes the nodes as
u = t^2 / (1 - t^2) and the weights w with sum(w) = F_0(x), the Boys function
(reference: src/rys_roots.rs:3036-3158, CINTrys_roots; src/g2e.rs:5649-5673
consumes u and w).

This script builds those rules from first principles, independently of the
reference's HONDO-style fits:

* exact rules: moments mu_k = F_k(x) (Boys function through the confluent
  hypergeometric function) of the weight in s = t^2, turned into the
  three-term recurrence by Gautschi's Chebyshev algorithm and solved by the
  Golub-Welsch eigenproblem, all in 60-digit mpmath;
* mid range 0 <= x < 43 + 5n: uniform segments of width H; on each segment
  every node u_i and weight w_i is interpolated at DEG+1 Chebyshev points and
  stored as monomial coefficients in the local variable
  t = (x - centre) / (H/2) in [-1, 1], evaluated by Horner's rule;
* large x >= 43 + 5n: the Gauss-Hermite limit t_i^2 = r_i / x,
  w_i = c_i * sqrt(pi / (4 x)), where r_i are the squared positive roots of
  H_{2n} and c_i their normalised weights.  The reference uses the same limit
  from 35 + 5n on (src/rys_roots.rs:3051); eight units later its truncation
  error, ~exp(-x) x^(2n-1), is below 1.2e-16 for every nroots here.

Every table is validated at random points against the exact rule; the
generator refuses to write a table whose worst relative error exceeds TOL.

Run:  python librint_b200/csrc/gen_rys_tables.py   (writes rys_tables.h)
"""
import multiprocessing
import os
import sys

from mpmath import mp, mpf, hyp1f1, matrix, eigsy, sqrt, cos, pi

DPS = 60
NMAX = 9          # nroots covered: (dd|dd) needs 5, its nuclear gradient 5,
                  # (ff|ff) 7, (gg|gg) 9
H = 4.0           # segment width in x
DEG = 18          # polynomial degree per segment (19 coefficients)
TOL = 2.0e-15     # worst accepted relative error of any node or weight
NVAL = 8          # validation points per segment
TOL_LARGEX = 2.0e-16  # worst accepted error of the large-x limit at xmax(n)


def xmax(n):
    # The reference switches to the large-x limit at 35 + 5n
    # (src/rys_roots.rs:3051), where the limit is still off by up to 6e-14
    # relative (nroots=9).  Eight more units of x bring it below 1.2e-16.
    return 43 + 5 * n


def boys(m, x):
    x = mpf(x)
    if x == 0:
        return mpf(1) / (2 * m + 1)
    return hyp1f1(m + mpf(1) / 2, m + mpf(3) / 2, -x) / (2 * m + 1)


def rys_rule(n, x):
    """Exact n-point rule at x: (u[0..n), w[0..n)) sorted by u ascending."""
    mp.dps = DPS
    mom = [boys(k, x) for k in range(2 * n)]
    sig_prev = [mpf(0)] * (2 * n)
    sig = list(mom)
    alpha = [mom[1] / mom[0]]
    beta = [mom[0]]
    for k in range(1, n):
        new = [mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha.append(new[k + 1] / new[k] - sig[k] / sig[k - 1])
        beta.append(new[k] / sig[k - 1])
        sig_prev, sig = sig, new
    jac = matrix(n, n)
    for i in range(n):
        jac[i, i] = alpha[i]
        if i + 1 < n:
            jac[i, i + 1] = jac[i + 1, i] = sqrt(beta[i + 1])
    ev, vec = eigsy(jac)
    pairs = sorted((ev[i], beta[0] * vec[0, i] ** 2) for i in range(n))
    u = [s / (1 - s) for s, _ in pairs]
    w = [wt for _, wt in pairs]
    return u, w


def _cheb_to_monomial(c):
    d = len(c) - 1
    tpoly = [[mpf(1)] + [mpf(0)] * d, [mpf(0), mpf(1)] + [mpf(0)] * (d - 1)]
    for j in range(2, d + 1):
        nt = [mpf(0)] * (d + 1)
        for i in range(d):
            nt[i + 1] += 2 * tpoly[j - 1][i]
        for i in range(d + 1):
            nt[i] -= tpoly[j - 2][i]
        tpoly.append(nt)
    mono = [mpf(0)] * (d + 1)
    for j in range(d + 1):
        for i in range(d + 1):
            mono[i] += c[j] * tpoly[j][i]
    return mono


def fit_segment(args):
    n, seg = args
    mp.dps = DPS
    a = mpf(seg) * mpf(H)
    b = a + mpf(H)
    nodes = [cos(pi * (k + mpf(1) / 2) / (DEG + 1)) for k in range(DEG + 1)]
    vals = []
    for t in nodes:
        u, w = rys_rule(n, (a + b) / 2 + (b - a) / 2 * t)
        vals.append(u + w)
    coefs = []
    for f in range(2 * n):
        c = []
        for j in range(DEG + 1):
            sm = sum(vals[k][f] * cos(pi * j * (k + mpf(1) / 2) / (DEG + 1))
                     for k in range(DEG + 1))
            c.append(sm * 2 / (DEG + 1) if j > 0 else sm / (DEG + 1))
        coefs.append([float(m) for m in _cheb_to_monomial(c)])
    # validation at pseudo-random interior points, evaluated in float64
    worst = 0.0
    for k in range(NVAL):
        frac = ((k * 0.6180339887498949 + seg * 0.31415926) % 1.0)
        x = float(a) + frac * H
        u, w = rys_rule(n, mpf(x))
        exact = u + w
        t = (x - (float(a) + H / 2)) / (H / 2)
        for f in range(2 * n):
            r = coefs[f][DEG]
            for i in range(DEG - 1, -1, -1):
                r = r * t + coefs[f][i]
            worst = max(worst, abs(float((mpf(r) - exact[f]) / exact[f])))
    return n, seg, coefs, worst


def large_x_constants(n):
    """Squared positive Hermite H_{2n} roots r_i and normalised weights c_i."""
    mp.dps = DPS
    # Gauss rule of exp(-y^2) on (-inf, inf) with 2n points via Golub-Welsch
    m = 2 * n
    jac = matrix(m, m)
    for i in range(m - 1):
        jac[i, i + 1] = jac[i + 1, i] = sqrt(mpf(i + 1) / 2)
    ev, vec = eigsy(jac)
    mu0 = sqrt(pi)
    pos = sorted((ev[i], mu0 * vec[0, i] ** 2) for i in range(m) if ev[i] > 0)
    r = [y * y for y, _ in pos]
    c = [wt / (sqrt(pi) / 2) for _, wt in pos]
    return r, c


def check_large_x(n, r, c):
    """Worst relative error of the large-x limit at the breakpoint."""
    x = mpf(xmax(n))
    u, w = rys_rule(n, x)
    worst = 0.0
    for i in range(n):
        ua = r[i] / (x - r[i])
        wa = c[i] * sqrt(pi / 4 / x)
        worst = max(worst, abs(float((ua - u[i]) / u[i])), abs(float((wa - w[i]) / w[i])))
    return worst


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rys_tables.h")
    jobs = []
    for n in range(1, NMAX + 1):
        nseg = int(-(-xmax(n) // H))
        jobs += [(n, s) for s in range(nseg)]
    ctx = multiprocessing.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        res = pool.map(fit_segment, jobs)
    table = {}
    for n, seg, coefs, worst in res:
        table[(n, seg)] = coefs
        if worst > TOL:
            sys.exit(f"fit failed: nroots={n} segment={seg} worst rel err {worst:.3e}")
    worst_by_n = {}
    for n, seg, _, worst in res:
        worst_by_n[n] = max(worst_by_n.get(n, 0.0), worst)
    lines = []
    lines.append("// Generated by gen_rys_tables.py -- do not edit.")
    lines.append("// Piecewise polynomial Rys nodes u=t^2/(1-t^2) and weights (sum = F_0(x)).")
    lines.append("// Layout per nroots n: [segment][function 0..2n)[coefficient 0..DEG],")
    lines.append("// functions 0..n-1 are u_i, n..2n-1 are w_i, ascending u; Horner in")
    lines.append("// t = (x - x_centre)/(H/2).  x >= 43+5n uses the large-x constants.")
    for n in range(1, NMAX + 1):
        lines.append(f"// nroots={n}: worst validated relative error {worst_by_n[n]:.2e}")
    lines.append("#pragma once")
    lines.append("// CUDA translation units define RYS_TAB_QUAL as __device__ and")
    lines.append("// RYS_CONST_QUAL as __constant__ before including this file.")
    lines.append("#ifndef RYS_TAB_QUAL")
    lines.append("#define RYS_TAB_QUAL")
    lines.append("#endif")
    lines.append("#ifndef RYS_CONST_QUAL")
    lines.append("#define RYS_CONST_QUAL")
    lines.append("#endif")
    lines.append(f"#define RYS_NMAX {NMAX}")
    lines.append(f"#define RYS_DEG {DEG}")
    lines.append(f"#define RYS_NCOEF {DEG + 1}")
    lines.append(f"#define RYS_SEG_WIDTH {H!r}")
    offs = [0]
    nsegs = []
    for n in range(1, NMAX + 1):
        nseg = int(-(-xmax(n) // H))
        nsegs.append(nseg)
        offs.append(offs[-1] + nseg * 2 * n * (DEG + 1))
    lines.append("static constexpr int RYS_TAB_NSEG[RYS_NMAX + 1] = {0, " +
                 ", ".join(str(s) for s in nsegs) + "};")
    lines.append("static constexpr int RYS_TAB_OFFSET[RYS_NMAX + 2] = {0, " +
                 ", ".join(str(o) for o in offs) + "};")
    lines.append("#ifndef RYS_OMIT_TAB   // translation units that take the table by pointer")
    lines.append(f"RYS_TAB_QUAL static const double RYS_TAB[{offs[-1]}] = {{")
    for n in range(1, NMAX + 1):
        for s in range(nsegs[n - 1]):
            for f in range(2 * n):
                lines.append("  " + ", ".join(repr(v) for v in table[(n, s)][f]) + ",")
    lines.append("};")
    lines.append("#endif")
    # large-x constants, packed per n at offset n(n-1)/2
    rr, cc, largex_err = [], [], []
    for n in range(1, NMAX + 1):
        r, c = large_x_constants(n)
        err = check_large_x(n, r, c)
        if err > TOL_LARGEX:
            sys.exit(f"large-x limit inaccurate at nroots={n}: {err:.3e}")
        largex_err.append(err)
        rr += [float(v) for v in r]
        cc += [float(v) for v in c]
    lines.append("// large-x limit, worst relative error at the breakpoint per nroots: " +
                 " ".join(f"{e:.1e}" for e in largex_err))
    lines.append(f"RYS_CONST_QUAL static const double RYS_LARGEX_R[{len(rr)}] = {{" +
                 ", ".join(repr(v) for v in rr) + "};")
    lines.append(f"RYS_CONST_QUAL static const double RYS_LARGEX_W[{len(cc)}] = {{" +
                 ", ".join(repr(v) for v in cc) + "};")
    with open(out, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    for n in range(1, NMAX + 1):
        print(f"nroots={n}: segments={nsegs[n-1]} worst rel err {worst_by_n[n]:.2e}")
    print("wrote", out, "doubles:", offs[-1])


if __name__ == "__main__":
    main()
