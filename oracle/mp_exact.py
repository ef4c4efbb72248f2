"""Extended-precision ERI for one shell quartet (test infrastructure only).

Used to triangulate disagreements between the double-precision paths and the
reference: the quartet is evaluated with exact Rys rules (60-digit Golub-
Welsch, ``librint_b200/csrc/gen_rys_tables.rys_rule``) and the same VRR/HRR
recurrences as src/eri.rs:263-399, all in mpmath at ``DPS`` digits, without
screening.  Cartesian output in libcint layout (i fastest).  Slow: meant for
a handful of quartets.
"""
from __future__ import annotations

import os
import sys

import numpy as np
from mpmath import mp, mpf, sqrt, exp, pi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "librint_b200", "csrc"))
import gen_rys_tables  # noqa: E402

DPS = 40


def _cart(l):
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def _fac_sp(l):
    if l == 0:
        return 1 / (2 * sqrt(pi))
    if l == 1:
        return sqrt(mpf(3) / (4 * pi))
    return mpf(1)


def eri_cart_exact(atm, bas, env, shls):
    mp.dps = DPS
    omega = mpf(float(env[8])) if len(env) > 8 else mpf(0)
    atm = np.asarray(atm).reshape(-1, 6)
    bas = np.asarray(bas).reshape(-1, 8)
    sh = []
    for s in shls:
        b = bas[s]
        l, k = int(b[1]), int(b[2])
        r = [mpf(float(v)) for v in env[atm[b[0], 1]:atm[b[0], 1] + 3]]
        a = [mpf(float(v)) for v in env[b[5]:b[5] + k]]
        c = [mpf(float(v)) for v in env[b[6]:b[6] + k]]
        sh.append((l, r, a, c))
    (li, ri, ai, ci), (lj, rj, aj, cj), (lk, rk, ak, ck), (ll, rl, al, cl) = sh
    nmax, mmax = li + lj, lk + ll
    nroots = (nmax + mmax) // 2 + 1
    common = 2 * pi ** 3 / sqrt(pi) * _fac_sp(li) * _fac_sp(lj) * _fac_sp(lk) * _fac_sp(ll)
    CI, CJ, CK, CL = _cart(li), _cart(lj), _cart(lk), _cart(ll)
    out = [mpf(0)] * (len(CI) * len(CJ) * len(CK) * len(CL))
    rirj = [ri[d] - rj[d] for d in range(3)]
    rkrl = [rk[d] - rl[d] for d in range(3)]
    rr_ij = sum(v * v for v in rirj)
    rr_kl = sum(v * v for v in rkrl)
    for lp in range(len(al)):
        for kp in range(len(ak)):
            akl = ak[kp] + al[lp]
            ekl = exp(-rr_kl * ak[kp] * al[lp] / akl)
            rkl = [(ak[kp] * rk[d] + al[lp] * rl[d]) / akl for d in range(3)]
            for jp in range(len(aj)):
                for ip in range(len(ai)):
                    aij = ai[ip] + aj[jp]
                    eij = exp(-rr_ij * ai[ip] * aj[jp] / aij)
                    rij = [(ai[ip] * ri[d] + aj[jp] * rj[d]) / aij for d in range(3)]
                    fac = common * ci[ip] * cj[jp] * ck[kp] * cl[lp] * eij * ekl
                    a1 = aij * akl
                    a0 = a1 / (aij + akl)
                    fac1 = sqrt(a0 / (a1 ** 3)) * fac
                    pq = [rij[d] - rkl[d] for d in range(3)]
                    x = a0 * sum(v * v for v in pq)
                    # range separation: erf (omega > 0) as nodes at theta x,
                    # erfc (omega < 0) as full minus erf; exact at DPS digits
                    nodes = []
                    if omega == 0:
                        us, ws = gen_rys_tables.rys_rule(nroots, x)
                        nodes = list(zip(us, ws))
                    else:
                        theta = omega * omega / (omega * omega + a0)
                        if omega < 0:
                            us, ws = gen_rys_tables.rys_rule(nroots, x)
                            nodes = list(zip(us, ws))
                        us, ws = gen_rys_tables.rys_rule(nroots, x * theta)
                        sgn = 1 if omega > 0 else -1
                        nodes += [(u * theta / (u + 1 - u * theta), sgn * w * sqrt(theta))
                                  for u, w in zip(us, ws)]
                    mp.dps = DPS
                    for u, w in nodes:
                        u2 = a0 * u
                        t4 = mpf(1) / 2 / (u2 * (aij + akl) + a1)
                        t5 = u2 * t4
                        b00, b10, b01 = t5, t5 + t4 * akl, t5 + t4 * aij
                        g = []
                        for d in range(3):
                            cn = rij[d] - rj[d] - 2 * t5 * akl * pq[d]
                            cm = rkl[d] - rl[d] + 2 * t5 * aij * pq[d]
                            # V[n][m] by the 2D recurrence, then binomial HRR
                            V = [[mpf(0)] * (mmax + 1) for _ in range(nmax + 1)]
                            V[0][0] = w * fac1 if d == 2 else mpf(1)
                            for n in range(nmax + 1):
                                for m in range(mmax + 1):
                                    if n == 0 and m == 0:
                                        continue
                                    if n > 0:
                                        v = cn * V[n - 1][m]
                                        if n > 1:
                                            v += (n - 1) * b10 * V[n - 2][m]
                                        if m > 0:
                                            v += m * b00 * V[n - 1][m - 1]
                                    else:
                                        v = cm * V[0][m - 1]
                                        if m > 1:
                                            v += (m - 1) * b01 * V[0][m - 2]
                                    V[n][m] = v
                            # G[(i,j),(k,l)] = sum_s C(i,s) (Rj-Ri)^(i-s) sum_t C(k,t) (Rl-Rk)^(k-t) V[j+s][l+t]
                            from math import comb
                            dij = rj[d] - ri[d]
                            dkl = rl[d] - rk[d]
                            G = {}
                            for i in range(li + 1):
                                for j in range(lj + 1):
                                    for k in range(lk + 1):
                                        for l in range(ll + 1):
                                            s_ = mpf(0)
                                            for s in range(i + 1):
                                                for t in range(k + 1):
                                                    s_ += (comb(i, s) * dij ** (i - s) * comb(k, t)
                                                           * dkl ** (k - t) * V[j + s][l + t])
                                            G[(i, j, k, l)] = s_
                            g.append(G)
                        idx = 0
                        for fl in CL:
                            for fk in CK:
                                for fj in CJ:
                                    for fi in CI:
                                        p = mpf(1)
                                        for d in range(3):
                                            p *= g[d][(fi[d], fj[d], fk[d], fl[d])]
                                        out[idx] += p
                                        idx += 1
    return np.array([float(v) for v in out])
