// Oracle: CPU restatement of librint's Rys-ERI / RHF path (test infrastructure
// only -- see oracle.h).  Citations are paths inside the reference project.
#include "oracle.h"

#include <quadmath.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../librint_b200/csrc/rys_tables.h"

namespace {

constexpr int ATM_SLOTS = 6;   // src/scf.rs:14
constexpr int BAS_SLOTS = 8;   // src/scf.rs:15
constexpr int LMAX = 4;        // same shell limit as src/eri.rs:10
constexpr int NCART_MAX = (LMAX + 1) * (LMAX + 2) / 2;
constexpr int NROOT_MAX = 2 * LMAX + 1;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
inline int nsph(int l) { return 2 * l + 1; }

// Angular normalisation libcint folds into s and p shells
// (src/g1e.rs:776-782): 1/sqrt(4 pi) and sqrt(3/(4 pi)).
double common_fac_sp(int l) {
  if (l == 0) return 0.5 / std::sqrt(M_PI);
  if (l == 1) return std::sqrt(3.0 / (4.0 * M_PI));
  return 1.0;
}

// Cartesian exponents in libcint order, x-major descending
// (src/eri.rs:31-50, src/cint_bas.rs:234).
struct CartComp {
  int n;
  int x[NCART_MAX], y[NCART_MAX], z[NCART_MAX];
  explicit CartComp(int l) : n(0) {
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) {
        x[n] = lx; y[n] = ly; z[n] = l - lx - ly; ++n;
      }
  }
};

// ---------------------------------------------------------------- Rys roots
// Two sources of the n-point Rys rule, selected by orc_set_rys_mode:
//   0 (default): the node/weight tables of librint_b200/csrc/rys_tables.h
//     (generated by librint_b200/csrc/gen_rys_tables.py, own fits to exact
//     60-digit rules) -- the tables the CUDA kernels read;
//   1: the rule computed here in binary128 from the measure itself, sharing
//     no table, generator or algorithm with the kernels (rys_rule_q below).
// Both return nodes u = t^2/(1-t^2) and weights summing to F_0(x), the
// convention of CINTrys_roots (src/rys_roots.rs:3036-3158).
std::atomic<int> g_rys_mode{0};

using f128 = __float128;

// 128-point Gauss-Legendre rule on [0, 1] in binary128 (Newton on the
// Legendre recurrence), built once.
constexpr int GL_M = 128;
struct GaussLegendre {
  f128 t[GL_M], w[GL_M];
  GaussLegendre() {
    for (int i = 0; i < GL_M; ++i) {
      f128 z = cosq(M_PIq * (i + 0.75Q) / (GL_M + 0.5Q)), dp = 0;
      for (int it = 0; it < 100; ++it) {
        f128 p0 = 1, p1 = z;
        for (int k = 2; k <= GL_M; ++k) {
          const f128 p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
          p0 = p1;
          p1 = p2;
        }
        dp = GL_M * (z * p1 - p0) / (z * z - 1);
        const f128 dz = p1 / dp;
        z -= dz;
        if (fabsq(dz) <= 1e-33Q * fabsq(z)) break;
      }
      t[i] = (1 - z) / 2;                                  // [-1, 1] -> [0, 1]
      w[i] = 1 / ((1 - z * z) * dp * dp);                  // 2 / (...) / 2
    }
  }
};

// n-point Gauss rule of dmu(s) = e^{-x s} s^{-1/2} / 2 ds on [0, 1] (the Rys
// measure in s = t^2; its moments are the Boys functions F_m(x)):
//  * the measure in t, e^{-x t^2} dt on [0, T], T = min(1, 12 / sqrt(x))
//    (beyond T the density is below e^{-144} of its peak), is discretised by
//    the Gauss-Legendre rule scaled to [0, T];
//  * the Stieltjes procedure gives the recurrence coefficients alpha_k,
//    beta_k of the monic polynomials in s orthogonal under that measure;
//  * the nodes are the eigenvalues of the Jacobi matrix, found by bisection
//    on its Sturm sequence (LDL^T negative counts), and the weights are the
//    Christoffel numbers 1 / sum_k pi_k(s_i)^2 / h_k.
void rys_rule_q(int n, double xd, double *u, double *w) {
  static const GaussLegendre gl;
  const f128 x = xd;
  const f128 T = x > 144 ? 12 / sqrtq(x) : f128(1);
  f128 s[GL_M], W[GL_M], p0[GL_M], p1[GL_M];
  for (int j = 0; j < GL_M; ++j) {
    const f128 t = T * gl.t[j];
    s[j] = t * t;
    W[j] = T * gl.w[j] * expq(-x * s[j]);
    p0[j] = 0;
    p1[j] = 1;
  }
  f128 alpha[10], beta[10], h[10];
  for (int k = 0; k < n; ++k) {
    f128 num = 0, den = 0;
    for (int j = 0; j < GL_M; ++j) {
      const f128 q = W[j] * p1[j] * p1[j];
      den += q;
      num += q * s[j];
    }
    h[k] = den;
    alpha[k] = num / den;
    beta[k] = k == 0 ? den : den / h[k - 1];
    if (k + 1 < n)
      for (int j = 0; j < GL_M; ++j) {
        const f128 p2 = (s[j] - alpha[k]) * p1[j] - (k == 0 ? f128(0) : beta[k]) * p0[j];
        p0[j] = p1[j];
        p1[j] = p2;
      }
  }
  // eigenvalues below lam: negative pivots of J - lam I
  auto below = [&](f128 lam) {
    int c = 0;
    f128 d = alpha[0] - lam;
    if (d < 0) ++c;
    for (int k = 1; k < n; ++k) {
      if (d == 0) d = 1e-4900Q;
      d = alpha[k] - lam - beta[k] / d;
      if (d < 0) ++c;
    }
    return c;
  };
  for (int i = 0; i < n; ++i) {
    f128 lo = 0, hi = T * T;
    for (int it = 0; it < 400 && hi - lo > 1e-34Q * hi; ++it) {
      const f128 mid = (lo + hi) / 2;
      if (below(mid) > i) hi = mid; else lo = mid;
    }
    const f128 si = (lo + hi) / 2;
    f128 a = 0, b = 1, sum = b * b / h[0];
    for (int k = 0; k + 1 < n; ++k) {
      const f128 c = (si - alpha[k]) * b - (k == 0 ? f128(0) : beta[k]) * a;
      a = b;
      b = c;
      sum += b * b / h[k + 1];
    }
    u[i] = (double)(si / (1 - si));
    w[i] = (double)(1 / sum);
  }
}

void rys_roots(int n, double x, double *u, double *w) {
  if (g_rys_mode.load(std::memory_order_relaxed)) return rys_rule_q(n, x, u, w);
  const double xbreak = 43.0 + 5.0 * n;
  if (x >= xbreak) {
    const int off = n * (n - 1) / 2;
    const double t = std::sqrt(M_PI / 4.0 / x);
    for (int i = 0; i < n; ++i) {
      const double r = RYS_LARGEX_R[off + i];
      u[i] = r / (x - r);
      w[i] = RYS_LARGEX_W[off + i] * t;
    }
    return;
  }
  int seg = (int)(x * (1.0 / RYS_SEG_WIDTH));
  if (seg >= RYS_TAB_NSEG[n]) seg = RYS_TAB_NSEG[n] - 1;
  if (seg < 0) seg = 0;
  const double t = (x - (seg * RYS_SEG_WIDTH + 0.5 * RYS_SEG_WIDTH)) * (2.0 / RYS_SEG_WIDTH);
  const double *c = RYS_TAB + RYS_TAB_OFFSET[n] + (size_t)seg * 2 * n * RYS_NCOEF;
  for (int f = 0; f < 2 * n; ++f) {
    const double *cf = c + f * RYS_NCOEF;
    double r = cf[RYS_DEG];
    for (int k = RYS_DEG - 1; k >= 0; --k) r = r * t + cf[k];
    if (f < n) u[f] = r; else w[f - n] = r;
  }
}

// ---------------------------------------------------------------- shells
struct Shell {
  int l, nprim, nctr;
  const double *r, *a, *c;   // centre, exponents, coefficients [ctr][prim]
};

Shell shell_of(int sh, const int *atm, const int *bas, const double *env) {
  const int *b = bas + BAS_SLOTS * sh;
  Shell s;
  s.l = b[1]; s.nprim = b[2]; s.nctr = b[3];
  s.r = env + atm[ATM_SLOTS * b[0] + 1];
  s.a = env + b[5];
  s.c = env + b[6];
  return s;
}

// log of the largest |coefficient| per primitive over the contractions
// (src/optimizer.rs:661-687, CINTOpt_log_max_pgto_coeff).
void log_maxc(const Shell &s, double *out) {
  for (int p = 0; p < s.nprim; ++p) {
    double m = 0.0;
    for (int c = 0; c < s.nctr; ++c) m = std::max(m, std::fabs(s.c[c * s.nprim + p]));
    out[p] = std::log(m);
  }
}

double sqr_dist(const double *a, const double *b) {
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}

// ---------------------------------------------------------------- 2e kernel
// Per root and axis the 2D table is built on the "base" centre of each pair
// and shifted to the partner by horizontal recurrence: the base of (ij) is i
// when li > lj, else j; of (kl) k when lk > ll, else l (libcint's choice,
// src/g2e.rs:113-181, which keeps the HRR short on the high-l centre).
// G[a][b][c][d]: a = power on the bra base A, b on its partner B, c on the
// ket base C, d on its partner D.

struct Quartet {
  Shell si, sj, sk, sl;
  int li, lj, lk, ll, nroots;
  bool ibase, kbase;
  int lA, lB, lC, lD, nab, ncd;
  const double *rA, *rB, *rC, *rD;
  double common_factor, expcutoff;
  double omega;   // env[8]: range separation (0 Coulomb, > 0 erf, < 0 erfc)
  double rirj[3], rkrl[3], rr_ij, rr_kl;
  double AB[3], CD[3];
  int sB, sC, sA;   // strides of G: index = ((a*(lB+1) + b)*(ncd+1) + c)*(lD+1) + d
};

Quartet make_quartet(const int *shls, const int *atm, const int *bas, const double *env) {
  Quartet q;
  q.si = shell_of(shls[0], atm, bas, env);
  q.sj = shell_of(shls[1], atm, bas, env);
  q.sk = shell_of(shls[2], atm, bas, env);
  q.sl = shell_of(shls[3], atm, bas, env);
  q.li = q.si.l; q.lj = q.sj.l; q.lk = q.sk.l; q.ll = q.sl.l;
  q.nroots = (q.li + q.lj + q.lk + q.ll) / 2 + 1;   // src/g2e.rs:100-101
  q.ibase = q.li > q.lj;
  q.kbase = q.lk > q.ll;
  q.lA = q.ibase ? q.li : q.lj; q.lB = q.ibase ? q.lj : q.li;
  q.lC = q.kbase ? q.lk : q.ll; q.lD = q.kbase ? q.ll : q.lk;
  q.rA = q.ibase ? q.si.r : q.sj.r; q.rB = q.ibase ? q.sj.r : q.si.r;
  q.rC = q.kbase ? q.sk.r : q.sl.r; q.rD = q.kbase ? q.sl.r : q.sk.r;
  q.nab = q.lA + q.lB;
  q.ncd = q.lC + q.lD;
  q.sC = q.lD + 1;
  q.sB = (q.ncd + 1) * q.sC;
  q.sA = (q.lB + 1) * q.sB;
  // 2 pi^3 / sqrt(pi) times the s/p angular factors (src/g2e.rs:74-82)
  q.common_factor = 2.0 * M_PI * M_PI * M_PI / std::sqrt(M_PI) *
                    common_fac_sp(q.li) * common_fac_sp(q.lj) *
                    common_fac_sp(q.lk) * common_fac_sp(q.ll);
  // src/g2e.rs:83-92 (the no-optimizer loop reads envs.expcutoff)
  q.expcutoff = env[0] == 0.0 ? 60.0 : std::max(40.0, env[0]) + 1.0;
  q.omega = env[8];
  for (int d = 0; d < 3; ++d) {
    q.rirj[d] = q.si.r[d] - q.sj.r[d];
    q.rkrl[d] = q.sk.r[d] - q.sl.r[d];
    q.AB[d] = q.rA[d] - q.rB[d];
    q.CD[d] = q.rC[d] - q.rD[d];
  }
  q.rr_ij = q.rirj[0] * q.rirj[0] + q.rirj[1] * q.rirj[1] + q.rirj[2] * q.rirj[2];
  q.rr_kl = q.rkrl[0] * q.rkrl[0] + q.rkrl[1] * q.rkrl[1] + q.rkrl[2] * q.rkrl[2];
  return q;
}

// One root: B00/B10/B01/C00/C0p (src/g2e.rs:5655-5673), 2D VRR on (A, C)
// (src/g2e.rs:316-506), HRR A->B and C->D (src/g2e.rs:507-909).  Element e
// of axis ax is at g[ax][e * rs]: the tables of all roots of a primitive
// quartet interleave (root innermost, as libcint's g arrays).
void g_one_root(double *g[3], int rs, const Quartet &q, double aij, double akl,
                double a0, double fac1, double u, double w,
                const double *rij, const double *rkl, const double *rijrkl) {
  const int sA = q.sA * rs, sB = q.sB * rs, sC = q.sC * rs, sD = rs;
  const int nab = q.nab, ncd = q.ncd;
  const double a1 = aij * akl;
  const double u2 = a0 * u;
  const double tmp4 = 0.5 / (u2 * (aij + akl) + a1);
  const double tmp5 = u2 * tmp4;
  const double tmp1 = 2.0 * tmp5;
  const double tmp2 = tmp1 * akl;
  const double tmp3 = tmp1 * aij;
  const double b00 = tmp5;
  const double b10 = tmp5 + tmp4 * akl;
  const double b01 = tmp5 + tmp4 * aij;
  for (int ax = 0; ax < 3; ++ax) {
    double *G = g[ax];
    const double cn = rij[ax] - q.rA[ax] - tmp2 * rijrkl[ax];
    const double cm = rkl[ax] - q.rC[ax] + tmp3 * rijrkl[ax];
    // V(n, m) lives at G[n][0][m][0]
    auto V = [&](int n, int m) -> double & { return G[n * sA + m * sC]; };
    V(0, 0) = ax == 2 ? w * fac1 : 1.0;
    for (int m = 1; m <= ncd; ++m) {
      double v = cm * V(0, m - 1);
      if (m > 1) v += (m - 1) * b01 * V(0, m - 2);
      V(0, m) = v;
    }
    for (int n = 1; n <= nab; ++n)
      for (int m = 0; m <= ncd; ++m) {
        double v = cn * V(n - 1, m);
        if (n > 1) v += (n - 1) * b10 * V(n - 2, m);
        if (m > 0) v += m * b00 * V(n - 1, m - 1);
        V(n, m) = v;
      }
    // bra HRR: (x-RB) = (x-RA) + (RA-RB)
    const double ab = q.AB[ax];
    for (int b = 1; b <= q.lB; ++b)
      for (int a = 0; a <= nab - b; ++a)
        for (int c = 0; c <= ncd; ++c)
          G[a * sA + b * sB + c * sC] = G[(a + 1) * sA + (b - 1) * sB + c * sC] +
                                        ab * G[a * sA + (b - 1) * sB + c * sC];
    const double cd = q.CD[ax];
    for (int a = 0; a <= q.lA; ++a)
      for (int b = 0; b <= q.lB; ++b)
        for (int d = 1; d <= q.lD; ++d)
          for (int c = 0; c <= ncd - d; ++c)
            G[a * sA + b * sB + c * sC + d * sD] = G[a * sA + b * sB + (c + 1) * sC + (d - 1) * sD] +
                                                   cd * G[a * sA + b * sB + c * sC + (d - 1) * sD];
  }
}

// Primitive-pair data of an ordered shell pair (A, B), index n = b * nA + a,
// with the reference's screening key (CINTset_pairdata,
// src/optimizer.rs:732-808):
//  * bra form (the pair in the i, j slots): cce, exp(-mu R^2) and the
//    product centre as ri + (aj / (ai + aj)) (rj - ri); entries failing the
//    cutoff get centre 1e18 and factor 0; returns true when none passes;
//  * ket form (the k, l slots): cce, exp(-mu R^2) and the product centre as
//    (ak rk + al rl) / (ak + al); entries failing the cutoff are skipped by
//    the primitive loop (factor and centre 0).
// Both forms restate the two ways src/cint2e.rs's loops compute them.
double pair_log_rr(const Shell &a, const Shell &b, double rr) {
  double lr = 1.7 - 1.5 * std::log(a.a[a.nprim - 1] + b.a[b.nprim - 1]);
  if (a.l + b.l > 0) lr += (a.l + b.l) * std::log(std::sqrt(rr) + 1.0);
  return lr;
}

bool pair_bra(const Shell &si, const Shell &sj, double rr, double expcutoff, double *cce,
              double *e, double *r) {
  double lci[32], lcj[32];
  log_maxc(si, lci);
  log_maxc(sj, lcj);
  const double log_rr = pair_log_rr(si, sj, rr);
  bool empty = true;
  for (int jp = 0; jp < sj.nprim; ++jp)
    for (int ip = 0; ip < si.nprim; ++ip) {
      const int n = jp * si.nprim + ip;
      const double inv = 1.0 / (si.a[ip] + sj.a[jp]);
      const double x = rr * si.a[ip] * sj.a[jp] * inv;
      cce[n] = x - log_rr - lci[ip] - lcj[jp];
      if (cce[n] < expcutoff) {
        empty = false;
        const double wj = sj.a[jp] * inv;
        for (int d = 0; d < 3; ++d) r[3 * n + d] = si.r[d] + wj * (sj.r[d] - si.r[d]);
        e[n] = std::exp(-x);
      } else {
        for (int d = 0; d < 3; ++d) r[3 * n + d] = 1e18;
        e[n] = 0.0;
      }
    }
  return empty;
}

void pair_ket(const Shell &sk, const Shell &sl, double rr, double expcutoff, double *cce,
              double *e, double *r) {
  double lck[32], lcl[32];
  log_maxc(sk, lck);
  log_maxc(sl, lcl);
  const double log_rr = pair_log_rr(sk, sl, rr);
  for (int lp = 0; lp < sl.nprim; ++lp)
    for (int kp = 0; kp < sk.nprim; ++kp) {
      const int m = lp * sk.nprim + kp;
      const double ak = sk.a[kp], al = sl.a[lp];
      const double akl = ak + al;
      const double x = rr * ak * al / akl;
      cce[m] = x - log_rr - lck[kp] - lcl[lp];
      if (cce[m] > expcutoff) {
        for (int d = 0; d < 3; ++d) r[3 * m + d] = 0.0;
        e[m] = 0.0;
        continue;
      }
      for (int d = 0; d < 3; ++d) r[3 * m + d] = (ak * sk.r[d] + al * sl.r[d]) / akl;
      e[m] = std::exp(-x);
    }
}

// Pair data of every ordered shell pair of a molecule, built once for the
// molecule-wide paths (Fock builds, energy, dense tensor), as the reference's
// integral2e / integral2e_fock build libcint's optimizer once
// (src/scf.rs:236-250, 333-343).  Per pair (I * nbas + J), np = KI KJ
// entries each of: bra cce, bra factor, bra centre (3), ket cce, ket factor,
// ket centre (3).
struct PairCache {
  int nbas = 0;
  std::vector<long long> off;
  std::vector<char> empty;
  std::vector<double> buf;
  const double *at(int i, int j) const { return buf.data() + off[(size_t)i * nbas + j]; }
};

double squared_distance(const double *a, const double *b) {
  const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return d0 * d0 + d1 * d1 + d2 * d2;
}

void build_pair_cache(PairCache &pc, const int *atm, const int *bas, int nbas, const double *env,
                      int nt) {
  pc.nbas = nbas;
  pc.off.assign((size_t)nbas * nbas + 1, 0);
  for (int i = 0; i < nbas; ++i)
    for (int j = 0; j < nbas; ++j)
      pc.off[(size_t)i * nbas + j + 1] =
          pc.off[(size_t)i * nbas + j] + 10LL * bas[BAS_SLOTS * i + 2] * bas[BAS_SLOTS * j + 2];
  pc.buf.assign((size_t)pc.off.back(), 0.0);
  pc.empty.assign((size_t)nbas * nbas, 0);
  const double expcutoff = env[0] == 0.0 ? 60.0 : std::max(40.0, env[0]) + 1.0;
#pragma omp parallel for schedule(dynamic, 8) num_threads(nt)
  for (int i = 0; i < nbas; ++i) {
    const Shell si = shell_of(i, atm, bas, env);
    for (int j = 0; j < nbas; ++j) {
      const Shell sj = shell_of(j, atm, bas, env);
      const size_t np = (size_t)si.nprim * sj.nprim;
      double *p = pc.buf.data() + pc.off[(size_t)i * nbas + j];
      const double rr = squared_distance(si.r, sj.r);
      pc.empty[(size_t)i * nbas + j] = pair_bra(si, sj, rr, expcutoff, p, p + np, p + 2 * np);
      pair_ket(si, sj, rr, expcutoff, p + 5 * np, p + 6 * np, p + 7 * np);
    }
  }
}

// Cartesian block for one quartet, any contraction pattern.  Loop nest and
// screening follow CINT2e_loop_nopt (src/cint2e.rs:36-465) with
// CINTset_pairdata (src/optimizer.rs:732-808); the recurrence and the gout
// root sum follow src/eri.rs:421-516 / src/cint2e.rs:2456, with the
// recurrence orientation of src/g2e.rs:113-181.
// out must hold ncart(i)*nctr_i * ... doubles; it is overwritten.
int eri_cart(double *out, const Quartet &q, const PairCache *pc = nullptr,
             const int *shls = nullptr) {
  const Shell &si = q.si, &sj = q.sj, &sk = q.sk, &sl = q.sl;
  const int nfi = ncart(q.li), nfj = ncart(q.lj), nfk = ncart(q.lk), nfl = ncart(q.ll);
  const int ni = nfi * si.nctr, nj = nfj * sj.nctr, nk = nfk * sk.nctr, nl = nfl * sl.nctr;
  const size_t ntot = (size_t)ni * nj * nk * nl;
  std::memset(out, 0, ntot * sizeof(double));

  // pair data for (ij) and (kl): from the molecule's cache, or computed here
  // into per-thread scratch (grown once: no allocation per quartet)
  static thread_local std::vector<double> pbuf, gbuf, prim;
  static thread_local std::vector<int> goff;
  const size_t npij = (size_t)si.nprim * sj.nprim, npkl = (size_t)sk.nprim * sl.nprim;
  const double *cceij, *eij, *rij, *kcce, *kexp, *krkl;
  bool empty;
  if (pc) {
    const double *b = pc->at(shls[0], shls[1]), *k = pc->at(shls[2], shls[3]);
    empty = pc->empty[(size_t)shls[0] * pc->nbas + shls[1]] != 0;
    cceij = b;
    eij = b + npij;
    rij = b + 2 * npij;
    kcce = k + 5 * npkl;
    kexp = k + 6 * npkl;
    krkl = k + 7 * npkl;
  } else {
    if (pbuf.size() < 5 * (npij + npkl)) pbuf.resize(5 * (npij + npkl));
    double *b = pbuf.data(), *k = b + 5 * npij;
    empty = pair_bra(si, sj, q.rr_ij, q.expcutoff, b, b + npij, b + 2 * npij);
    cceij = b;
    eij = b + npij;
    rij = b + 2 * npij;
    if (!empty) pair_ket(sk, sl, q.rr_kl, q.expcutoff, k, k + npkl, k + 2 * npkl);
    kcce = k;
    kexp = k + npkl;
    krkl = k + 2 * npkl;
  }
  if (empty) return 0;

  const CartComp ci(q.li), cj(q.lj), ck(q.lk), cl(q.ll);
  const int nf = nfi * nfj * nfk * nfl;
  const int nc = si.nctr * sj.nctr * sk.nctr * sl.nctr;
  // per root three tables (x, y, z) of gs doubles each, all roots of a
  // primitive quartet side by side
  const int gs = (q.nab + 1) * q.sA;
  if (gbuf.size() < 3 * (size_t)gs * 2 * NROOT_MAX) gbuf.resize(3 * (size_t)gs * 2 * NROOT_MAX);
  if (prim.size() < (size_t)nf) {
    prim.resize(nf);
    goff.resize(3 * (size_t)nf);
  }
  // offsets into the per-axis tables of every cartesian element (i fastest):
  // G[a][b][c][d] with a, b the powers on the bra base and partner, c, d on
  // the ket's (src/g2e.rs:195-315, CINTg2e_index_xyz)
  {
    int idx = 0;
    for (int lf = 0; lf < nfl; ++lf)
      for (int kf = 0; kf < nfk; ++kf)
        for (int jf = 0; jf < nfj; ++jf)
          for (int iff = 0; iff < nfi; ++iff, ++idx) {
            const int pi_[3] = {ci.x[iff], ci.y[iff], ci.z[iff]};
            const int pj_[3] = {cj.x[jf], cj.y[jf], cj.z[jf]};
            const int pk_[3] = {ck.x[kf], ck.y[kf], ck.z[kf]};
            const int pl_[3] = {cl.x[lf], cl.y[lf], cl.z[lf]};
            for (int ax = 0; ax < 3; ++ax) {
              const int a = q.ibase ? pi_[ax] : pj_[ax], b = q.ibase ? pj_[ax] : pi_[ax];
              const int c = q.kbase ? pk_[ax] : pl_[ax], d = q.kbase ? pl_[ax] : pk_[ax];
              goff[3 * idx + ax] = a * q.sA + b * q.sB + c * q.sC + d;
            }
          }
  }
  const int *go = goff.data();
  double u[2 * NROOT_MAX], w[2 * NROOT_MAX];
  int any = 0;

  for (int lp = 0; lp < sl.nprim; ++lp) {
    const double al = sl.a[lp];
    for (int kp = 0; kp < sk.nprim; ++kp) {
      const double ak = sk.a[kp];
      const double akl = ak + al;
      const int m = lp * sk.nprim + kp;
      const double ccekl = kcce[m];
      if (ccekl > q.expcutoff) continue;
      const double *rkl = krkl + 3 * m;
      const double eijcutoff = q.expcutoff - ccekl;
      const double ekl = kexp[m];
      for (int jp = 0; jp < sj.nprim; ++jp)
        for (int ip = 0; ip < si.nprim; ++ip) {
          const int n = jp * si.nprim + ip;
          if (cceij[n] > eijcutoff) continue;
          const double aij = si.a[ip] + sj.a[jp];
          const double *pij = &rij[3 * n];
          const double fac = q.common_factor * eij[n] * ekl;
          // CINTg0_2e prefactors (src/g2e.rs:5563-5568)
          const double a1 = aij * akl;
          const double a0 = a1 / (aij + akl);
          const double fac1 = std::sqrt(a0 / (a1 * a1 * a1)) * fac;
          double rijrkl[3];
          for (int d = 0; d < 3; ++d) rijrkl[d] = pij[d] - rkl[d];
          const double x = a0 * (rijrkl[0] * rijrkl[0] + rijrkl[1] * rijrkl[1] +
                                 rijrkl[2] * rijrkl[2]);
          // range separation (src/g2e.rs:5564-5612): erf(omega r)/r for
          // omega > 0 through nodes at theta x mapped u -> u theta/(u + 1 -
          // u theta) and sqrt(theta) on the prefactor; erfc for omega < 0 as
          // the full operator minus the long-range one (second node set,
          // weights times -sqrt(theta)), skipped when theta x > 40 or beyond
          // the screening budget.  (The reference solves dedicated
          // short-range nodes for Rys orders >= 4; the two forms are the same
          // quadrature and differ by rounding.)
          int nr = q.nroots;
          double fac1r = fac1;
          if (q.omega == 0.0) {
            rys_roots(nr, x, u, w);
          } else {
            const double theta = q.omega * q.omega / (q.omega * q.omega + a0);
            if (q.omega > 0.0) {
              rys_roots(nr, x * theta, u, w);
              for (int r = 0; r < nr; ++r) u[r] = u[r] * theta / (u[r] + 1.0 - u[r] * theta);
              fac1r *= std::sqrt(theta);
            } else {
              if (theta * x > eijcutoff - cceij[n] || theta * x > 40.0) continue;
              rys_roots(nr, x, u, w);
              rys_roots(nr, x * theta, u + nr, w + nr);
              for (int r = nr; r < 2 * nr; ++r) {
                u[r] = u[r] * theta / (u[r] + 1.0 - u[r] * theta);
                w[r] *= -std::sqrt(theta);
              }
              nr *= 2;
            }
          }
          // every root's tables (root innermost), then per element the sum
          // over the roots in root order (CINTgout2e, src/cint2e.rs:2456-2895)
          double *gb = gbuf.data();
          const size_t ga = (size_t)gs * nr;     // one axis, all roots
          for (int r = 0; r < nr; ++r) {
            double *gr[3] = {gb + r, gb + ga + r, gb + 2 * ga + r};
            g_one_root(gr, nr, q, aij, akl, a0, fac1r, u[r], w[r], pij, rkl, rijrkl);
          }
          // segmented shells (one contraction each): the block is the
          // element order itself, so each element is contracted as it is summed
          const bool seg = nc == 1;
          const double cc1 = seg ? si.c[ip] * sj.c[jp] * sk.c[kp] * sl.c[lp] : 0.0;
          double *pr = prim.data();
          for (int idx = 0; idx < nf; ++idx) {
            const double *px = gb + (size_t)go[3 * idx] * nr;
            const double *py = gb + ga + (size_t)go[3 * idx + 1] * nr;
            const double *pz = gb + 2 * ga + (size_t)go[3 * idx + 2] * nr;
            double sum = 0.0;
            for (int r = 0; r < nr; ++r) {
              double v = px[r];
              v *= py[r];
              v *= pz[r];
              sum += v;
            }
            if (seg) out[idx] += cc1 * sum; else pr[idx] = sum;
          }
          any = 1;
          if (seg) continue;
          // contract over every (ci, cj, ck, cl) combination
          for (int c = 0; c < nc; ++c) {
            const int cci = c % si.nctr, ccj = (c / si.nctr) % sj.nctr;
            const int cck = (c / (si.nctr * sj.nctr)) % sk.nctr;
            const int ccl = c / (si.nctr * sj.nctr * sk.nctr);
            const double cc = si.c[cci * si.nprim + ip] * sj.c[ccj * sj.nprim + jp] *
                              sk.c[cck * sk.nprim + kp] * sl.c[ccl * sl.nprim + lp];
            int idx2 = 0;
            for (int lf = 0; lf < nfl; ++lf)
              for (int kf = 0; kf < nfk; ++kf)
                for (int jf = 0; jf < nfj; ++jf)
                  for (int iff = 0; iff < nfi; ++iff, ++idx2) {
                    const size_t o = (size_t)(iff + nfi * cci) +
                                     (size_t)ni * ((jf + nfj * ccj) +
                                     (size_t)nj * ((kf + nfk * cck) + (size_t)nk * (lf + nfl * ccl)));
                    out[o] += cc * prim[idx2];
                  }
          }
        }
    }
  }
  return any;
}

// ---------------------------------------------------------------- cart2sph
// Real solid harmonics in libcint order and normalisation (m = -l..l; p kept
// as x, y, z).  Coefficients from the closed form of Helgaker, Jorgensen &
// Olsen, "Molecular Electronic-Structure Theory", eqs. 6.4.47-6.4.50, scaled
// by sqrt((2l+1)/(4 pi)); the reference tabulates the same numbers
// (src/cart2sph.rs:26, d shells at :88463-88538).
double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}
double fact(int n) { double r = 1.0; for (int i = 2; i <= n; ++i) r *= i; return r; }

struct SphTable {
  // c[l][ms][cart]: coefficient of cartesian component cart in sph function ms
  std::vector<double> c[LMAX + 1];
  SphTable() {
    for (int l = 0; l <= LMAX; ++l) {
      const int nc = ncart(l), ns = nsph(l);
      c[l].assign(ns * nc, 0.0);
      if (l <= 1) {
        for (int i = 0; i < nc; ++i) c[l][i * nc + i] = 1.0;
        continue;
      }
      const CartComp cc(l);
      const double scale = std::sqrt((2 * l + 1) / (4.0 * M_PI));
      for (int m = -l; m <= l; ++m) {
        const int am = std::abs(m);
        const double norm = 1.0 / (std::pow(2.0, am) * fact(l)) *
                            std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
        const int twovm = m < 0 ? 1 : 0;   // 2 v_m
        for (int t = 0; t <= (l - am) / 2; ++t)
          for (int uu = 0; uu <= t; ++uu)
            for (int twov = twovm; twov <= am; twov += 2) {
              // v = twov/2; v runs v_m .. floor(|m|/2 - v_m) + v_m
              const int sgn_exp = t + (twov - twovm) / 2;
              const double coef = (sgn_exp % 2 ? -1.0 : 1.0) * std::pow(0.25, t) * binom(l, t) *
                                  binom(l - t, am + t) * binom(t, uu) * binom(am, twov);
              const int px = 2 * t + am - 2 * uu - twov;
              const int py = 2 * uu + twov;
              const int pz = l - 2 * t - am;
              for (int k = 0; k < nc; ++k)
                if (cc.x[k] == px && cc.y[k] == py && cc.z[k] == pz)
                  c[l][(m + l) * nc + k] += norm * scale * coef;
            }
      }
    }
  }
};
const SphTable &sph_table() { static SphTable t; return t; }

// Transform a cartesian block (i fastest, nctr folded in) to spherical
// (src/cart2sph.rs:90199-90282 transforms j, l, k, then i; the order only
// changes rounding).
void cart2sph_4(double *sph, const double *cart, const Quartet &q) {
  const int l4[4] = {q.li, q.lj, q.lk, q.ll};
  const int nct[4] = {q.si.nctr, q.sj.nctr, q.sk.nctr, q.sl.nctr};
  int dim[4];
  for (int a = 0; a < 4; ++a) dim[a] = ncart(l4[a]) * nct[a];
  std::vector<double> cur(cart, cart + (size_t)dim[0] * dim[1] * dim[2] * dim[3]);
  for (int ax = 0; ax < 4; ++ax) {
    const int l = l4[ax], nc = ncart(l), ns = nsph(l);
    const std::vector<double> &co = sph_table().c[l];
    int ndim[4] = {dim[0], dim[1], dim[2], dim[3]};
    ndim[ax] = ns * nct[ax];
    size_t inner = 1, outer = 1;
    for (int a = 0; a < ax; ++a) inner *= dim[a];
    for (int a = ax + 1; a < 4; ++a) outer *= dim[a];
    std::vector<double> nxt(inner * ndim[ax] * outer, 0.0);
    for (size_t o = 0; o < outer; ++o)
      for (int ct = 0; ct < nct[ax]; ++ct)
        for (int m = 0; m < ns; ++m)
          for (int k = 0; k < nc; ++k) {
            const double cf = co[m * nc + k];
            if (cf == 0.0) continue;
            const double *src = &cur[(o * dim[ax] + ct * nc + k) * inner];
            double *dst = &nxt[(o * ndim[ax] + ct * ns + m) * inner];
            for (size_t i = 0; i < inner; ++i) dst[i] += cf * src[i];
          }
    cur.swap(nxt);
    dim[ax] = ndim[ax];
  }
  std::memcpy(sph, cur.data(), cur.size() * sizeof(double));
}

int quartet_block(double *out, int coord, const int *shls, const int *atm,
                  const int *bas, const double *env, const PairCache *pc = nullptr) {
  const Quartet q = make_quartet(shls, atm, bas, env);
  if (coord == 0) return eri_cart(out, q, pc, shls);
  const size_t nct = (size_t)ncart(q.li) * q.si.nctr * ncart(q.lj) * q.sj.nctr *
                     ncart(q.lk) * q.sk.nctr * ncart(q.ll) * q.sl.nctr;
  std::vector<double> cart(nct);
  const int r = eri_cart(cart.data(), q, pc, shls);
  cart2sph_4(out, cart.data(), q);
  return r;
}

int shell_dim(int coord, const int *bas, int sh) {
  const int l = bas[BAS_SLOTS * sh + 1], nctr = bas[BAS_SLOTS * sh + 3];
  return (coord == 0 ? ncart(l) : nsph(l)) * nctr;
}

std::vector<int> shell_offsets(int coord, const int *bas, int nbas) {
  std::vector<int> off(nbas + 1, 0);
  for (int s = 0; s < nbas; ++s) off[s + 1] = off[s] + shell_dim(coord, bas, s);
  return off;
}

int threads_or_default(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

// ---------------------------------------------------------------- 1e
// Primitive-pair 1D overlaps by the Obara-Saika recurrence; kinetic as
// -1/2 d^2/dx^2 on the ket; nuclear attraction by Rys quadrature with
// (li+lj)/2+1 roots per point nucleus.  Same operators and normalisation as
// cint1e_ovlp/kin/nuc_cart (src/cint1e.rs:925,976; src/intor1.rs:168;
// src/g1e.rs:241-330).
void overlap_1d(double *s, int imax, int jmax, double xpa, double xpb, double oo2p) {
  // s[i*(jmax+1)+j], s(0,0) = 1
  const int ld = jmax + 1;
  s[0] = 1.0;
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      double v;
      if (i > 0) {
        v = xpa * s[(i - 1) * ld + j];
        if (i > 1) v += oo2p * (i - 1) * s[(i - 2) * ld + j];
        if (j > 0) v += oo2p * j * s[(i - 1) * ld + j - 1];
      } else {
        v = xpb * s[j - 1];
        if (j > 1) v += oo2p * (j - 1) * s[j - 2];
      }
      s[i * ld + j] = v;
    }
}

void int1e_block(double *out, int typec, const Shell &a, const Shell &b,
                 const int *atm, int natm, const double *env) {
  const int la = a.l, lb = b.l, nfa = ncart(la), nfb = ncart(lb);
  const int na = nfa * a.nctr, nb = nfb * b.nctr;
  std::memset(out, 0, sizeof(double) * na * nb);
  const CartComp ca(la), cb(lb);
  const double rab2 = sqr_dist(a.r, b.r);
  const double cfac = common_fac_sp(la) * common_fac_sp(lb);
  const int imax = la, jmax = lb + (typec == 1 ? 2 : 0);
  double sx[3][(LMAX + 1) * (LMAX + 3)];
  std::vector<double> prim(nfa * nfb);
  for (int jp = 0; jp < b.nprim; ++jp)
    for (int ip = 0; ip < a.nprim; ++ip) {
      const double ai = a.a[ip], bj = b.a[jp], p = ai + bj;
      const double mu = ai * bj / p;
      const double eab = std::exp(-mu * rab2);
      double P[3];
      for (int d = 0; d < 3; ++d) P[d] = (ai * a.r[d] + bj * b.r[d]) / p;
      std::fill(prim.begin(), prim.end(), 0.0);
      if (typec == 0 || typec == 1) {
        for (int d = 0; d < 3; ++d)
          overlap_1d(sx[d], imax, jmax, P[d] - a.r[d], P[d] - b.r[d], 0.5 / p);
        const double pre = cfac * eab * std::pow(M_PI / p, 1.5);
        const int ld = jmax + 1;
        for (int jf = 0; jf < nfb; ++jf)
          for (int iff = 0; iff < nfa; ++iff) {
            const int ia[3] = {ca.x[iff], ca.y[iff], ca.z[iff]};
            const int jb[3] = {cb.x[jf], cb.y[jf], cb.z[jf]};
            double v;
            if (typec == 0) {
              v = sx[0][ia[0] * ld + jb[0]] * sx[1][ia[1] * ld + jb[1]] * sx[2][ia[2] * ld + jb[2]];
            } else {
              v = 0.0;
              for (int d = 0; d < 3; ++d) {
                const int j = jb[d];
                const double *s = sx[d] + ia[d] * ld;
                double t = -2.0 * bj * (2 * j + 1) * s[j] + 4.0 * bj * bj * s[j + 2];
                if (j >= 2) t += j * (j - 1) * s[j - 2];
                t *= -0.5;
                double o = 1.0;
                for (int e = 0; e < 3; ++e)
                  if (e != d) o *= sx[e][ia[e] * ld + jb[e]];
                v += t * o;
              }
            }
            prim[iff + nfa * jf] = pre * v;
          }
      } else {
        const int nroots = (la + lb) / 2 + 1;
        double u[NROOT_MAX], w[NROOT_MAX];
        const int lsum = la + lb;
        double ix[3][LMAX * 2 + 1][LMAX + 1];
        for (int c = 0; c < natm; ++c) {
          const int *ac = atm + ATM_SLOTS * c;
          const double *rc = env + ac[1];
          const double z = -std::fabs((double)ac[0]);
          const double pc2 = sqr_dist(P, rc);
          rys_roots(nroots, p * pc2, u, w);
          const double pre = cfac * eab * 2.0 * M_PI / p * z;
          for (int r = 0; r < nroots; ++r) {
            const double t2 = u[r] / (1.0 + u[r]);
            for (int d = 0; d < 3; ++d) {
              // 1D: I(n+1) = (PA - t2 PC) I(n) + n/(2p) (1-t2) I(n-1), then HRR to j
              double g[2 * LMAX + 2];
              g[0] = 1.0;
              const double c0 = (P[d] - a.r[d]) - t2 * (P[d] - rc[d]);
              const double b1 = 0.5 / p * (1.0 - t2);
              if (lsum > 0) g[1] = c0;
              for (int n = 1; n < lsum; ++n) g[n + 1] = c0 * g[n] + n * b1 * g[n - 1];
              // HRR: I(i, j+1) = I(i+1, j) + (A-B) I(i, j)
              double h[2 * LMAX + 2][LMAX + 1];
              for (int i = 0; i <= lsum; ++i) h[i][0] = g[i];
              const double ab = a.r[d] - b.r[d];
              for (int j = 1; j <= lb; ++j)
                for (int i = 0; i <= lsum - j; ++i) h[i][j] = h[i + 1][j - 1] + ab * h[i][j - 1];
              for (int i = 0; i <= la; ++i)
                for (int j = 0; j <= lb; ++j) ix[d][i][j] = h[i][j];
            }
            for (int jf = 0; jf < nfb; ++jf)
              for (int iff = 0; iff < nfa; ++iff)
                prim[iff + nfa * jf] += pre * w[r] * ix[0][ca.x[iff]][cb.x[jf]] *
                                        ix[1][ca.y[iff]][cb.y[jf]] * ix[2][ca.z[iff]][cb.z[jf]];
          }
        }
      }
      for (int cj = 0; cj < b.nctr; ++cj)
        for (int cI = 0; cI < a.nctr; ++cI) {
          const double cc = a.c[cI * a.nprim + ip] * b.c[cj * b.nprim + jp];
          for (int jf = 0; jf < nfb; ++jf)
            for (int iff = 0; iff < nfa; ++iff)
              out[(iff + nfa * cI) + na * (jf + nfb * cj)] += cc * prim[iff + nfa * jf];
        }
    }
}

// 2-index cart -> sph for a 1e block (i fastest)
void cart2sph_2(double *sph, const double *cart, const Shell &a, const Shell &b) {
  const int nca = ncart(a.l), ncb = ncart(b.l), nsa = nsph(a.l), nsb = nsph(b.l);
  const int Na = nca * a.nctr, Nb = ncb * b.nctr, Sa = nsa * a.nctr;
  const std::vector<double> &A = sph_table().c[a.l], &B = sph_table().c[b.l];
  std::vector<double> tmp((size_t)Sa * Nb, 0.0);
  for (int j = 0; j < Nb; ++j)
    for (int ct = 0; ct < a.nctr; ++ct)
      for (int m = 0; m < nsa; ++m) {
        double v = 0.0;
        for (int k = 0; k < nca; ++k) v += A[m * nca + k] * cart[(ct * nca + k) + Na * j];
        tmp[(ct * nsa + m) + Sa * j] = v;
      }
  for (int i = 0; i < Sa; ++i)
    for (int ct = 0; ct < b.nctr; ++ct)
      for (int m = 0; m < nsb; ++m) {
        double v = 0.0;
        for (int k = 0; k < ncb; ++k) v += B[m * ncb + k] * tmp[i + Sa * (ct * ncb + k)];
        sph[i + Sa * (ct * nsb + m)] = v;
      }
}

// ---------------------------------------------------------------- linear algebra
// Cyclic Jacobi eigensolver for a symmetric matrix (row-major, overwritten).
// Eigenvalues ascending in w, eigenvectors in the columns of V (row-major).
void eigh(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double a2 = A[(size_t)i * n + j] * A[(size_t)i * n + j];
        tot += a2;
        if (i != j) off += a2;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - s * akq;
          A[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - s * aqk;
          A[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - s * vkq;
          V[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[(size_t)i * n + i];
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return w[x] < w[y]; });
  std::vector<double> w2(n), V2((size_t)n * n);
  for (int c = 0; c < n; ++c) {
    w2[c] = w[idx[c]];
    for (int r = 0; r < n; ++r) V2[(size_t)r * n + c] = V[(size_t)r * n + idx[c]];
  }
  w.swap(w2);
  V.swap(V2);
}

std::vector<double> matmul(int n, const std::vector<double> &A, const std::vector<double> &B) {
  std::vector<double> C((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      const double a = A[(size_t)i * n + k];
      for (int j = 0; j < n; ++j) C[(size_t)i * n + j] += a * B[(size_t)k * n + j];
    }
  return C;
}

double nuclear_repulsion(const int *atm, int natm, const double *env) {
  double e = 0.0;
  for (int i = 0; i < natm; ++i)
    for (int j = 0; j < i; ++j) {
      const double *ri = env + atm[ATM_SLOTS * i + 1], *rj = env + atm[ATM_SLOTS * j + 1];
      e += (double)(atm[ATM_SLOTS * i] * atm[ATM_SLOTS * j]) / std::sqrt(sqr_dist(ri, rj));
    }
  return e;
}

}  // namespace

// ====================================================================== C API
extern "C" {

void orc_rys_roots(int n, double x, double *u, double *w) { rys_roots(n, x, u, w); }
void orc_set_rys_mode(int mode) { g_rys_mode.store(mode ? 1 : 0); }

int orc_nao(int coord, const int *bas, int nbas) {
  int n = 0;
  for (int s = 0; s < nbas; ++s) n += shell_dim(coord, bas, s);
  return n;
}

int orc_int2e_cart(double *out, const int *shls, const int *atm, int, const int *bas,
                   int, const double *env) {
  return quartet_block(out, 0, shls, atm, bas, env);
}

int orc_int2e_sph(double *out, const int *shls, const int *atm, int, const int *bas,
                  int, const double *env) {
  return quartet_block(out, 1, shls, atm, bas, env);
}

void orc_int2e_batch(double *out, int coord, const int *shls, long nq, const int *atm,
                     int, const int *bas, int, const double *env, int nthreads) {
  std::vector<size_t> off(nq + 1, 0);
  for (long q = 0; q < nq; ++q) {
    size_t d = 1;
    for (int a = 0; a < 4; ++a) d *= shell_dim(coord, bas, shls[4 * q + a]);
    off[q + 1] = off[q] + d;
  }
  const int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
  for (long q = 0; q < nq; ++q) quartet_block(out + off[q], coord, shls + 4 * q, atm, bas, env);
}

void orc_int2e_tensor(double *out, int coord, const int *atm, int, const int *bas,
                      int nbas, const double *env, int nthreads) {
  const std::vector<int> off = shell_offsets(coord, bas, nbas);
  const size_t n = off[nbas];
  const int nt = threads_or_default(nthreads);
  PairCache pc;
  build_pair_cache(pc, atm, bas, nbas, env, nt);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> buf;
#pragma omp for schedule(dynamic) collapse(2)
    for (int i = 0; i < nbas; ++i)
      for (int j = 0; j < nbas; ++j)
        for (int k = 0; k < nbas; ++k)
          for (int l = 0; l < nbas; ++l) {
            const int shls[4] = {i, j, k, l};
            const int di = off[i + 1] - off[i], dj = off[j + 1] - off[j];
            const int dk = off[k + 1] - off[k], dl = off[l + 1] - off[l];
            buf.resize((size_t)di * dj * dk * dl);
            quartet_block(buf.data(), coord, shls, atm, bas, env, &pc);
            size_t c = 0;
            for (int L = 0; L < dl; ++L)
              for (int K = 0; K < dk; ++K)
                for (int J = 0; J < dj; ++J)
                  for (int I = 0; I < di; ++I, ++c)
                    out[(((size_t)(off[i] + I) * n + off[j] + J) * n + off[k] + K) * n + off[l] + L] = buf[c];
          }
  }
}

void orc_int1e(double *out, int coord, int typec, const int *atm, int natm, const int *bas,
               int nbas, const double *env) {
  const std::vector<int> off = shell_offsets(coord, bas, nbas);
  const int n = off[nbas];
  std::vector<double> cart, sph;
  for (int i = 0; i < nbas; ++i)
    for (int j = 0; j < nbas; ++j) {
      const Shell a = shell_of(i, atm, bas, env), b = shell_of(j, atm, bas, env);
      cart.resize((size_t)ncart(a.l) * a.nctr * ncart(b.l) * b.nctr);
      int1e_block(cart.data(), typec, a, b, atm, natm, env);
      const double *blk = cart.data();
      if (coord == 1) {
        sph.resize((size_t)nsph(a.l) * a.nctr * nsph(b.l) * b.nctr);
        cart2sph_2(sph.data(), cart.data(), a, b);
        blk = sph.data();
      }
      const int di = off[i + 1] - off[i], dj = off[j + 1] - off[j];
      for (int J = 0; J < dj; ++J)
        for (int I = 0; I < di; ++I) out[(size_t)(off[i] + I) * n + off[j] + J] = blk[I + di * J];
    }
}

void orc_fock_G(double *G, const double *P, int coord, const int *atm, int, const int *bas,
                int nbas, const double *env, int nthreads) {
  const std::vector<int> off = shell_offsets(coord, bas, nbas);
  const size_t n = off[nbas];
  std::memset(G, 0, n * n * sizeof(double));
  const int nt = threads_or_default(nthreads);
  PairCache pc;
  build_pair_cache(pc, atm, bas, nbas, env, nt);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> Gl(n * n, 0.0), buf;
#pragma omp for schedule(dynamic) collapse(2)
    for (int i = 0; i < nbas; ++i)
      for (int j = 0; j < nbas; ++j)
        for (int k = 0; k < nbas; ++k)
          for (int l = 0; l < nbas; ++l) {
            const int shls[4] = {i, j, k, l};
            const int di = off[i + 1] - off[i], dj = off[j + 1] - off[j];
            const int dk = off[k + 1] - off[k], dl = off[l + 1] - off[l];
            buf.resize((size_t)di * dj * dk * dl);
            quartet_block(buf.data(), coord, shls, atm, bas, env, &pc);
            size_t c = 0;
            // slot (mu nu | sig lam): G[mu,nu] += P[lam,sig] v; G[mu,lam] -= P[nu,sig] v / 2
            // (src/scf.rs:379-391)
            for (int L = 0; L < dl; ++L)
              for (int K = 0; K < dk; ++K)
                for (int J = 0; J < dj; ++J)
                  for (int I = 0; I < di; ++I, ++c) {
                    const size_t mu = off[i] + I, nu = off[j] + J, sg = off[k] + K, lm = off[l] + L;
                    const double v = buf[c];
                    Gl[mu * n + nu] += P[lm * n + sg] * v;
                    Gl[mu * n + lm] += -0.5 * P[nu * n + sg] * v;
                  }
          }
#pragma omp critical
    for (size_t x = 0; x < n * n; ++x) G[x] += Gl[x];
  }
}

// One quartet's digestion, the reference's loop body (src/scf.rs:379-391):
// slot (mu nu | sig lam): G[mu,nu] += P[lam,sig] v; G[mu,lam] -= P[nu,sig] v / 2.
static void digest_quartet(double *G, const double *P, size_t n, const std::vector<int> &off,
                           const int shls[4], const double *buf) {
  const int i = shls[0], j = shls[1], k = shls[2], l = shls[3];
  const int di = off[i + 1] - off[i], dj = off[j + 1] - off[j];
  const int dk = off[k + 1] - off[k], dl = off[l + 1] - off[l];
  size_t c = 0;
  for (int L = 0; L < dl; ++L)
    for (int K = 0; K < dk; ++K)
      for (int J = 0; J < dj; ++J)
        for (int I = 0; I < di; ++I, ++c) {
          const size_t mu = off[i] + I, nu = off[j] + J, sg = off[k] + K, lm = off[l] + L;
          const double v = buf[c];
          G[mu * n + nu] += P[lm * n + sg] * v;
          G[mu * n + lm] += -0.5 * P[nu * n + sg] * v;
        }
}

void orc_fock_G_quartets(double *G, const double *P, const int *shls, long nq, const int *atm,
                         int, const int *bas, int nbas, const double *env, int nthreads) {
  const std::vector<int> off = shell_offsets(0, bas, nbas);
  const size_t n = off[nbas];
  std::memset(G, 0, n * n * sizeof(double));
  const int nt = threads_or_default(nthreads);
  PairCache pc;
  build_pair_cache(pc, atm, bas, nbas, env, nt);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> Gl(n * n, 0.0), buf;
#pragma omp for schedule(dynamic, 64)
    for (long q = 0; q < nq; ++q) {
      const int *s4 = shls + 4 * q;
      size_t d = 1;
      for (int a = 0; a < 4; ++a) d *= off[s4[a] + 1] - off[s4[a]];
      buf.resize(d);
      quartet_block(buf.data(), 0, s4, atm, bas, env, &pc);
      digest_quartet(Gl.data(), P, n, off, s4, buf.data());
    }
#pragma omp critical
    for (size_t x = 0; x < n * n; ++x) G[x] += Gl[x];
  }
}

void orc_fock_G_blocks(double *out, const double *P, const int *pairs, int npairs,
                       const int *atm, int, const int *bas, int nbas, const double *env,
                       int nthreads) {
  const std::vector<int> off = shell_offsets(0, bas, nbas);
  const size_t n = off[nbas];
  std::vector<size_t> boff(npairs + 1, 0);
  for (int p = 0; p < npairs; ++p)
    boff[p + 1] = boff[p] + (size_t)(off[pairs[2 * p] + 1] - off[pairs[2 * p]]) *
                                (off[pairs[2 * p + 1] + 1] - off[pairs[2 * p + 1]]);
  std::memset(out, 0, boff[npairs] * sizeof(double));
  const int nt = threads_or_default(nthreads);
  PairCache pc;
  build_pair_cache(pc, atm, bas, nbas, env, nt);
  // Block (X, Y): every quartet of the reference's nbas^4 loop whose digestion
  // touches G[mu in X, nu in Y]: (X Y | K L) through the first update and
  // (X J | K Y) through the second.
  for (int p = 0; p < npairs; ++p) {
    const int X = pairs[2 * p], Y = pairs[2 * p + 1];
    const int dx = off[X + 1] - off[X], dy = off[Y + 1] - off[Y];
#pragma omp parallel num_threads(nt)
    {
      std::vector<double> loc((size_t)dx * dy, 0.0), buf;
#pragma omp for schedule(dynamic) collapse(2)
      for (int a = 0; a < nbas; ++a)
        for (int b = 0; b < nbas; ++b) {
          for (int pass = 0; pass < 2; ++pass) {
            // pass 0: (X Y | a b), G[mu,nu] += P[lam,sig] v
            // pass 1: (X a | b Y), G[mu,lam] -= P[nu,sig] v / 2
            const int s4[4] = {X, pass == 0 ? Y : a, pass == 0 ? a : b, pass == 0 ? b : Y};
            const int d0 = off[s4[0] + 1] - off[s4[0]], d1 = off[s4[1] + 1] - off[s4[1]];
            const int d2 = off[s4[2] + 1] - off[s4[2]], d3 = off[s4[3] + 1] - off[s4[3]];
            buf.resize((size_t)d0 * d1 * d2 * d3);
            quartet_block(buf.data(), 0, s4, atm, bas, env, &pc);
            size_t c = 0;
            for (int L = 0; L < d3; ++L)
              for (int K = 0; K < d2; ++K)
                for (int J = 0; J < d1; ++J)
                  for (int I = 0; I < d0; ++I, ++c) {
                    const size_t nu = off[s4[1]] + J, sg = off[s4[2]] + K, lm = off[s4[3]] + L;
                    if (pass == 0)
                      loc[(size_t)I * dy + J] += P[lm * n + sg] * buf[c];
                    else
                      loc[(size_t)I * dy + L] += -0.5 * P[nu * n + sg] * buf[c];
                  }
          }
        }
#pragma omp critical
      for (size_t x = 0; x < (size_t)dx * dy; ++x) out[boff[p] + x] += loc[x];
    }
  }
}

double orc_energy2_sym(const double *P, const int *atm, int, const int *bas, int nbas,
                       const double *env, int nthreads) {
  // 1/2 sum P G(P) over unique quartets: with the 8-fold permutational
  // symmetry of (ab|cd) and a symmetric P, 1/2 sum_{abcd} (ab|cd)
  // [P_ab P_cd - 1/4 (P_ac P_bd + P_ad P_bc)] equals 1/2 tr(P G(P)) of the
  // reference's digestion (src/scf.rs:379-391); each unique shell quartet
  // carries its degeneracy weight.
  const std::vector<int> off = shell_offsets(0, bas, nbas);
  const size_t n = off[nbas];
  const long npair = (long)nbas * (nbas + 1) / 2;
  std::vector<int> pi(npair), pj(npair);
  for (int i = 0, p = 0; i < nbas; ++i)
    for (int j = 0; j <= i; ++j, ++p) { pi[p] = i; pj[p] = j; }
  double total = 0.0;
  const int nt = threads_or_default(nthreads);
  PairCache pc;
  build_pair_cache(pc, atm, bas, nbas, env, nt);
#pragma omp parallel num_threads(nt) reduction(+ : total)
  {
    std::vector<double> buf;
#pragma omp for schedule(dynamic, 1)
    for (long bra = npair - 1; bra >= 0; --bra) {
      const int i = pi[bra], j = pj[bra];
      double acc = 0.0;
      for (long ket = 0; ket <= bra; ++ket) {
        const int k = pi[ket], l = pj[ket];
        const int s4[4] = {i, j, k, l};
        const int di = off[i + 1] - off[i], dj = off[j + 1] - off[j];
        const int dk = off[k + 1] - off[k], dl = off[l + 1] - off[l];
        buf.resize((size_t)di * dj * dk * dl);
        if (!quartet_block(buf.data(), 0, s4, atm, bas, env, &pc)) continue;
        const double w = (i != j ? 2.0 : 1.0) * (k != l ? 2.0 : 1.0) * (bra != ket ? 2.0 : 1.0);
        double s = 0.0;
        size_t c = 0;
        for (int L = 0; L < dl; ++L)
          for (int K = 0; K < dk; ++K)
            for (int J = 0; J < dj; ++J)
              for (int I = 0; I < di; ++I, ++c) {
                const size_t a = off[i] + I, b = off[j] + J, cc = off[k] + K, d = off[l] + L;
                s += buf[c] * (P[a * n + b] * P[cc * n + d] -
                               0.25 * (P[a * n + cc] * P[b * n + d] + P[a * n + d] * P[b * n + cc]));
              }
        acc += w * s;
      }
      total += acc;
    }
  }
  return 0.5 * total;
}

double orc_energy1(const double *P, const int *atm, int natm, const int *bas, int nbas,
                   const double *env) {
  const int n = orc_nao(0, bas, nbas);
  const size_t nn = (size_t)n * n;
  std::vector<double> T(nn), V(nn);
  orc_int1e(T.data(), 0, 1, atm, natm, bas, nbas, env);
  orc_int1e(V.data(), 0, 2, atm, natm, bas, nbas, env);
  double e1 = 0.0;
  for (size_t x = 0; x < nn; ++x) e1 += P[x] * (T[x] + V[x]);
  return e1 + nuclear_repulsion(atm, natm, env);
}

int orc_density(double *Pout, size_t nelec, int imax, double conv, const int *atm, int natm,
                const int *bas, int nbas, const double *env, int nthreads, int *iters) {
  const int n = orc_nao(0, bas, nbas);
  const size_t nn = (size_t)n * n;
  std::vector<double> S(nn), T(nn), V(nn), H(nn), G(nn);
  orc_int1e(S.data(), 0, 0, atm, natm, bas, nbas, env);
  orc_int1e(T.data(), 0, 1, atm, natm, bas, nbas, env);
  orc_int1e(V.data(), 0, 2, atm, natm, bas, nbas, env);
  for (size_t x = 0; x < nn; ++x) H[x] = T[x] + V[x];
  // find_X (src/scf.rs:607-649): X = U s^-1/2, refuse s_min < 1e-8
  std::vector<double> s, U;
  eigh(n, S, s, U);
  if (s[0] < 1e-8) return 1;
  std::vector<double> X(nn), Xt(nn);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) X[(size_t)r * n + c] = U[(size_t)r * n + c] / std::sqrt(s[c]);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) Xt[(size_t)c * n + r] = X[(size_t)r * n + c];
  // P = I (src/scf.rs:757-764); plain Roothaan iteration (src/scf.rs:774-784)
  std::vector<double> P(nn, 0.0), Pold;
  for (int i = 0; i < n; ++i) P[(size_t)i * n + i] = 1.0;
  double delta = 1.0;
  int it = 0;
  while (delta > conv && it < imax) {
    Pold = P;
    orc_fock_G(G.data(), P.data(), 0, atm, natm, bas, nbas, env, nthreads);
    std::vector<double> F(nn);
    for (size_t x = 0; x < nn; ++x) F[x] = H[x] + G[x];
    std::vector<double> Fp = matmul(n, matmul(n, Xt, F), X);
    std::vector<double> e, Uf;
    eigh(n, Fp, e, Uf);
    std::vector<double> C = matmul(n, X, Uf);
    std::fill(P.begin(), P.end(), 0.0);
    for (int mu = 0; mu < n; ++mu)
      for (int nu = 0; nu < n; ++nu) {
        double v = 0.0;
        for (size_t i = 0; i < nelec / 2; ++i) v += 2.0 * C[(size_t)mu * n + i] * C[(size_t)nu * n + i];
        P[(size_t)mu * n + nu] = v;
      }
    double d = 0.0;
    for (size_t x = 0; x < nn; ++x) d += (P[x] - Pold[x]) * (P[x] - Pold[x]);
    delta = std::sqrt(d) / 2.0;
    ++it;
  }
  if (iters) *iters = it;
  if (delta > conv) return 2;
  // check_density (src/scf.rs:572-600)
  double tr = 0.0;
  for (int mu = 0; mu < n; ++mu)
    for (int nu = 0; nu < n; ++nu) tr += P[(size_t)mu * n + nu] * S[(size_t)nu * n + mu];
  if (std::fabs(tr - (double)nelec) > 1e-6) return 3;
  std::vector<double> PSP = matmul(n, matmul(n, P, S), P);
  double idem = 0.0;
  for (size_t x = 0; x < nn; ++x) idem = std::max(idem, std::fabs(PSP[x] - 2.0 * P[x]));
  if (idem > 1e-6) return 3;
  std::memcpy(Pout, P.data(), nn * sizeof(double));
  return 0;
}

double orc_energy(const double *P, const int *atm, int natm, const int *bas, int nbas,
                  const double *env, int nthreads) {
  // energyfast (src/scf.rs:827-956): sum P (T+V) + 1/2 sum P G(P) + E_nn
  const int n = orc_nao(0, bas, nbas);
  const size_t nn = (size_t)n * n;
  std::vector<double> T(nn), V(nn), G(nn);
  orc_int1e(T.data(), 0, 1, atm, natm, bas, nbas, env);
  orc_int1e(V.data(), 0, 2, atm, natm, bas, nbas, env);
  orc_fock_G(G.data(), P, 0, atm, natm, bas, nbas, env, nthreads);
  double e1 = 0.0, e2 = 0.0;
  for (size_t x = 0; x < nn; ++x) {
    e1 += P[x] * (T[x] + V[x]);
    e2 += 0.5 * P[x] * G[x];
  }
  return e1 + e2 + nuclear_repulsion(atm, natm, env);
}

double orc_scf(size_t nelec, int imax, double conv, const int *atm, int natm, const int *bas,
               int nbas, const double *env, int nthreads) {
  const int n = orc_nao(0, bas, nbas);
  std::vector<double> P((size_t)n * n);
  if (orc_density(P.data(), nelec, imax, conv, atm, natm, bas, nbas, env, nthreads, nullptr) != 0)
    return NAN;
  return orc_energy(P.data(), atm, natm, bas, nbas, env, nthreads);
}

}  // extern "C"
