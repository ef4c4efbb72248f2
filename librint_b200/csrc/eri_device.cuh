// Device side of the Rys-quadrature ERI engine (sm_100a, FP64).
//
// Work decomposition for one angular class (LI LJ | LK LL), canonical order
// LI >= LJ, LK >= LL, (LI,LJ) >= (LK,LL):
//
//  * The recurrence is built on the "base" centre of each pair (i if LI > LJ,
//    else j; k if LK > LL, else l) as libcint does (reference
//    src/g2e.rs:113-181).  A = bra base, B = bra partner, C/D likewise.
//  * Per primitive quartet only the Rys roots, the 2D VRR table V(n, m),
//    n <= LA+LB, m <= LC+LD, and the (e|f) product sum run:
//        [e|f] += sum_r Vx_r[ex][fx] Vy_r[ey][fy] Vz_r[ez][fz]
//    over cartesian e of momentum LA..LA+LB on A and f of LC..LC+LD on C.
//    The horizontal recurrences (A->B, C->D) and the cart->sph transform are
//    linear with shell-quartet constants, so they run once per contracted
//    shell quartet in the epilogue ("HRR after contraction").
//  * A warp holds SLOTS = 32 / NROW shell quartets; within a slot lane rho
//    owns row e = rho of [e|f] and keeps its NCOL f-accumulators in
//    registers.  Roots and VRR are computed cooperatively by the slot's
//    lanes and exchanged through a small per-warp shared-memory area.
//  * Roots/weights come from the piecewise polynomial tables of
//    rys_tables.h, staged once per CTA in shared memory.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rys_tables.h"

namespace lrb {

// ------------------------------------------------------------------ shapes
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nsph(int l) { return 2 * l + 1; }

// cartesian component n of momentum l in libcint order (x-major descending)
__host__ __device__ constexpr int cart_x(int l, int n) {
  int c = 0;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      if (c == n) return lx;
      ++c;
    }
  return 0;
}
__host__ __device__ constexpr int cart_y(int l, int n) {
  int c = 0;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      if (c == n) return ly;
      ++c;
    }
  return 0;
}
__host__ __device__ constexpr int cart_z(int l, int n) { return l - cart_x(l, n) - cart_y(l, n); }
// position of (x, y, z) inside momentum x+y+z
__host__ __device__ constexpr int cart_index(int x, int y, int z) {
  return (y + z) * (y + z + 1) / 2 + z;
}
// components of all momenta lo..hi, concatenated
__host__ __device__ constexpr int range_count(int lo, int hi) {
  int n = 0;
  for (int e = lo; e <= hi; ++e) n += ncart(e);
  return n;
}
__host__ __device__ constexpr int range_offset(int lo, int e) {
  int n = 0;
  for (int k = lo; k < e; ++k) n += ncart(k);
  return n;
}
__host__ __device__ constexpr int range_x(int lo, int r) {
  int e = lo;
  while (r >= ncart(e)) { r -= ncart(e); ++e; }
  return cart_x(e, r);
}
__host__ __device__ constexpr int range_y(int lo, int r) {
  int e = lo;
  while (r >= ncart(e)) { r -= ncart(e); ++e; }
  return cart_y(e, r);
}
__host__ __device__ constexpr int range_z(int lo, int r) {
  int e = lo;
  while (r >= ncart(e)) { r -= ncart(e); ++e; }
  return cart_z(e, r);
}
__host__ __device__ constexpr int range_index(int lo, int x, int y, int z) {
  return range_offset(lo, x + y + z) + cart_index(x, y, z);
}
__host__ __device__ constexpr int binom(int n, int k) {
  int r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// Component ax (0, 1, 2) of a 3-vector held in registers.  Indexing a local
// array with a runtime axis would place it on the stack (local memory).
template <typename T>
__device__ __forceinline__ T pick3(T x, T y, T z, int ax) {
  return ax == 0 ? x : (ax == 1 ? y : z);
}

// ------------------------------------------------------------------ data
// One primitive pair of a shell pair: exponent sum, Gaussian product centre,
// coefficient product times exp(-mu R^2) (class prefactor folded into the
// ket side by the caller), and libcint's screening key
// cce = mu R^2 - log_rr - log|c_i| - log|c_j| (reference
// src/optimizer.rs:732-808).
// ia = 1/a and facia = fac/a let the kernels form the prefactor
// sqrt(a0/(a_ij a_kl)^3) fac_ij fac_kl = sqrt(1/(a_ij+a_kl)) facia_ij facia_kl
// and the recurrence coefficients without divisions.
struct __align__(16) PrimPair {
  double a, ia, px, py, pz, fac, facia, cce;
};

// One shell quartet of a class launch, canonical order.
struct QuartetJob {
  int pij_off, nij;       // bra primitive pairs
  int pkl_off, nkl;       // ket primitive pairs
  int ish, jsh, ksh, lsh; // canonical shells (centres)
  long long out_off;      // first output element
  int s_i, s_j, s_k, s_l; // output strides of the canonical indices
};

// Sort key of a primitive pair's screening value: NaN orders last.
__device__ __forceinline__ double cce_key(double c) { return c != c ? INFINITY : c; }

// A shell pair of a molecule's pair table (oriented l_i >= l_j).
struct PairInfo {
  int ish, jsh;           // shells
  int pp_off, npp;        // primitive pairs in the PrimPair array
};

// Fock-build extras: density and the unsymmetrised accumulators
// (G = J + J^T - (K + K^T)/2 is formed afterwards).
struct FockParams {
  const int2 *jobs;       // (bra pair, ket pair) with bra class >= ket class
  const PairInfo *pairs;
  const int *aooff;       // first AO of each shell
  const double *P;        // n x n row-major
  double *J, *K;          // n x n accumulators
  int n;
  // measurement only: when not NULL, the launch adds the number of primitive
  // quartets that passed screening (one atomic per warp at its end)
  unsigned long long *prim_count;
  // primitive screening (when lq is not NULL): a primitive quartet is skipped
  // when Q_bra Q_ket d < tau_prim, with Q the primitive pairs' Schwarz
  // factors (log, float) and d the quartet's density factor from Dsh
  const float *lq;
  double tau_prim;
  const double *Dsh;      // shell-block maxima of |P|, nbas x nbas
  int nbas;
};

struct EriParams {
  const QuartetJob *jobs;
  const int *order;       // jobs to run, in launch order
  int njobs;
  const PrimPair *pp;
  const double *centers;  // 3 doubles per shell
  double *out;
  double expcutoff;       // env[0] == 0 ? 60 : max(40, env[0]) + 1 (reference src/g2e.rs:83-92)
  double omega;           // env[8]: 0 Coulomb, > 0 long range (erf), < 0 short range (erfc)
  int sph;                // 1: spherical output, 0: cartesian
};

// ------------------------------------------------------------------ roots
// Table geometry (segments of width 4 up to 43 + 5n), usable in device code.
__host__ __device__ constexpr int rys_nseg(int n) { return (43 + 5 * n + 3) / 4; }
__host__ __device__ constexpr int rys_tab_offset(int n) {
  int o = 0;
  for (int k = 1; k < n; ++k) o += rys_nseg(k) * 2 * k * RYS_NCOEF;
  return o;
}
static_assert(rys_tab_offset(5) == RYS_TAB_OFFSET[5] && rys_tab_offset(10) == RYS_TAB_OFFSET[10] &&
                  rys_nseg(9) == RYS_TAB_NSEG[9],
              "table geometry out of sync with rys_tables.h");

// Rys nodes/weights for N roots at x from the shared-memory table `tab`
// (layout of rys_tables.h for this N).  Function f < N is u_f, f >= N is
// w_{f-N}.
template <int N>
__device__ __forceinline__ double rys_function(const double *tab, double x, int f) {
  constexpr double XBREAK = 43.0 + 5.0 * N;
  if (x >= XBREAK) {
    constexpr int off = N * (N - 1) / 2;
    if (f < N) {
      const double r = RYS_LARGEX_R[off + f];
      return r / (x - r);
    }
    return RYS_LARGEX_W[off + f - N] * sqrt(0.78539816339744831 / x);  // pi/4
  }
  // clamp keeps the table read in bounds even for NaN input (NaN propagates)
  constexpr int NSEG = rys_nseg(N);
  static_assert(RYS_SEG_WIDTH == 4.0, "segment count assumes width 4");
  int seg = (int)(x * (1.0 / RYS_SEG_WIDTH));
  seg = seg < 0 ? 0 : (seg >= NSEG ? NSEG - 1 : seg);
  const double t = (x - (seg * RYS_SEG_WIDTH + 0.5 * RYS_SEG_WIDTH)) * (2.0 / RYS_SEG_WIDTH);
  const double *c = tab + (seg * 2 * N + f) * RYS_NCOEF;
  double r = c[RYS_DEG];
#pragma unroll
  for (int k = RYS_DEG - 1; k >= 0; --k) r = fma(r, t, c[k]);
  return r;
}

}  // namespace lrb
