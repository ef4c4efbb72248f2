// Adjoint ERI kernel: the two-electron part of the frozen-density gradient
// with respect to basis exponents and contraction coefficients (the
// reference's dRf, src/dscf.rs:370-515, which reverse-differentiates
// src/eri.rs:eri_cart with Enzyme).
//
// For one canonical shell quartet (IJ|KL) with degeneracy weight w and
//   Gamma_abcd = 4 P_ab P_cd - P_ac P_bd - P_ad P_bc
// the quartet's share of dE_2e/dtheta is w sum_abcd Gamma_abcd dI_abcd/dtheta
// (the 8 permutation images folded in).  A job puts the differentiated shell
// X first, (X Y | Z W), so the derivative always acts on position i:
//   d/dc_p : primitive p of X only, divided by c_p   (RAISE = 0)
//   d/da_p : d/da (c x^a e^{-a r^2}) = -c r^2 x^a e^{-a r^2}, i.e. the class
//            with l_X + 2 contracted with -sum_axis Gamma(a' - 2e_axis) (MODE 2).
//   d/dX_d : d/dX_d (x^a e^{-a r^2}) = 2 a_p x^(a+e_d) e^.. - a_d x^(a-e_d) e^..,
//            the class with l_X + 1 contracted per axis with Gamma(a' - e_d)
//            and weighted by 2 a_p (MODE 1), and the class with l_X - 1
//            contracted with -(a'_d + 1) Gamma(a' + e_d) (MODE 3); the three
//            axis sums go to the atom of X (nuclear-coordinate gradient).
// Primitives of X are the outer loop, so every primitive gets one reduced
// scalar; the recurrences and the root handling are those of the energy
// kernel (vrr_hrr_unit, rys_function).
#pragma once
#include "eri_kernel.cuh"

namespace lrb {

constexpr int GRAD_WARPS = 2;
constexpr int GRAD_THREADS = 32 * GRAD_WARPS;

struct GradJob {
  int bp, kp;       // pair holding X (X first), the other pair
  int xsecond;      // X is the second shell of pair bp
  int pad;
};

struct GradParams {
  const GradJob *jobs;
  const int *order;
  int njobs;
  const PairInfo *pairs;
  const PrimPair *pp;
  const double *centers;
  const int *bas;
  const int *aooff;
  const double *env;
  const double *P;
  int n;
  double expcutoff;
  double *grad;     // d/d env[s1 + t] (modes 0, 2)
  int s1;
  double *gatom;    // d/d atom coordinates, 3 per atom (modes 1, 3)
};

// modes: 0 coefficient, 2 exponent, 1 and 3 the raised and lowered parts of
// the centre derivative; dl is the momentum change of X, nc the axis sums
__host__ __device__ constexpr int grad_dl(int mode) { return mode == 3 ? -1 : mode; }
__host__ __device__ constexpr int grad_nc(int mode) { return (mode == 1 || mode == 3) ? 3 : 1; }

template <class C, int NC = 1>
struct GradLayout {
  static constexpr int LOOP = 3 * C::NR + C::NR * 3 * C::GSZ + C::NR * 3 * C::TSZ;
  static constexpr int GAM1 = C::NBRA * C::NKET;   // one Gamma table
  static constexpr int GAM = NC * GAM1;
  static constexpr int RED = 32 * NC;
  static constexpr int SLOT = LOOP + GAM + RED;
  static constexpr int WARP = C::SLOTS * SLOT;
  static constexpr int TAB = (RYS_TAB_OFFSET[C::NR + 1] - RYS_TAB_OFFSET[C::NR]);
  static constexpr size_t SMEM = sizeof(double) * (size_t)(TAB + GRAD_WARPS * WARP);
};

// S[c] += sum_k gam[c * stride + k] x[col_x(k)] y[col_y(k)] z[col_z(k)]
template <class C, int NC, int STRIDE, int K>
__device__ __forceinline__ void gout_gamma(double (&S)[NC], const double *gam,
                                           const double (&x)[C::CW], const double (&y)[C::CW],
                                           const double (&z)[C::CW]) {
  if constexpr (K < C::NCOLS) {
    constexpr int X = C::col_off(K, 0), Y = C::col_off(K, 1), Z = C::col_off(K, 2);
    const double t = x[X] * y[Y] * z[Z];
#pragma unroll
    for (int c = 0; c < NC; ++c) S[c] = fma(gam[c * STRIDE + K], t, S[c]);
    gout_gamma<C, NC, STRIDE, K + 1>(S, gam, x, y, z);
  }
}

__device__ __forceinline__ int cart_pos(int x, int y, int z) {
  return (y + z) * (y + z + 1) / 2 + z;
}

template <int LX, int LY, int LZ, int LW, int MODE>
__global__ void __launch_bounds__(GRAD_THREADS)
k_eri_grad(GradParams gp, const double *__restrict__ rys_tab_n, int *counter) {
  constexpr int NC = grad_nc(MODE);
  using C = EriClass<LX + grad_dl(MODE), LY, LZ, LW>;
  using L = GradLayout<C, NC>;
  extern __shared__ double smem[];
  double *tab = smem;
  for (int i = threadIdx.x; i < L::TAB; i += blockDim.x) tab[i] = rys_tab_n[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *wbuf = smem + L::TAB + warp * L::WARP;
  const int slot = lane / C::LANES;
  const int rho = lane - slot * C::LANES;
  const bool lane_live = slot < C::SLOTS;
  const int myslot = lane_live ? slot : C::SLOTS - 1;
  double *sb = wbuf + myslot * L::SLOT;
  double *RW = sb;
  double *G = sb + 3 * C::NR;
  double *Tsc = G + C::NR * 3 * C::GSZ;
  double *Gam = sb + L::LOOP;              // [rows][cols]
  double *red = Gam + L::GAM;              // per-lane partial sums

  int roff[3] = {0, 0, 0};
  {
    const int r = rho < C::NROWS ? rho : 0;
    const int p = C::ROWKET ? C::NK : C::NI;
    const int lp = C::ROWKET ? C::LK : C::LI, lq = C::ROWKET ? C::LL : C::LJ;
    int px, py, pz, qx, qy, qz;
    cart_comp_rt(lp, r % p, px, py, pz);
    cart_comp_rt(lq, r / p, qx, qy, qz);
    const int pc[3] = {px, py, pz}, qc[3] = {qx, qy, qz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      if (C::ROWKET) {
        const int c = C::KB ? pc[ax] : qc[ax], d = C::KB ? qc[ax] : pc[ax];
        roff[ax] = (c * (C::LD + 1) + d) * C::BSZ;
      } else {
        const int a = C::IB ? pc[ax] : qc[ax], b = C::IB ? qc[ax] : pc[ax];
        roff[ax] = (a * (C::LB + 1) + b) * C::KSZ;
      }
    }
  }
  int xrow[C::NEX > 0 ? C::NEX : 1], xcol[C::NEX > 0 ? C::NEX : 1], xoff[C::NEX > 0 ? C::NEX : 1][3];
  if constexpr (C::NEX > 0) {
#pragma unroll
    for (int k = 0; k < C::NEX; ++k) {
      const int e = lane + 32 * k;
      xrow[k] = e < C::EXTRA ? 32 + e / C::NCOLS : -1;
      xcol[k] = e < C::EXTRA ? e % C::NCOLS : 0;
      const int row = e < C::EXTRA ? 32 + e / C::NCOLS : 0;
      const int p = C::ROWKET ? C::NK : C::NI;
      const int lp = C::ROWKET ? C::LK : C::LI, lq = C::ROWKET ? C::LL : C::LJ;
      const int cp = C::ROWKET ? C::NI : C::NK;
      const int lcp = C::ROWKET ? C::LI : C::LK, lcq = C::ROWKET ? C::LJ : C::LL;
      int px, py, pz, qx, qy, qz, ux, uy, uz, vx, vy, vz;
      cart_comp_rt(lp, row % p, px, py, pz);
      cart_comp_rt(lq, row / p, qx, qy, qz);
      cart_comp_rt(lcp, xcol[k] % cp, ux, uy, uz);
      cart_comp_rt(lcq, xcol[k] / cp, vx, vy, vz);
      const int pc[3] = {px, py, pz}, qc[3] = {qx, qy, qz}, uc[3] = {ux, uy, uz}, vc[3] = {vx, vy, vz};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        if (C::ROWKET) {
          const int c = C::KB ? pc[ax] : qc[ax], d = C::KB ? qc[ax] : pc[ax];
          const int a = C::IB ? uc[ax] : vc[ax], b = C::IB ? vc[ax] : uc[ax];
          xoff[k][ax] = (c * (C::LD + 1) + d) * C::BSZ + a * (C::LB + 1) + b;
        } else {
          const int a = C::IB ? pc[ax] : qc[ax], b = C::IB ? qc[ax] : pc[ax];
          const int c = C::KB ? uc[ax] : vc[ax], d = C::KB ? vc[ax] : uc[ax];
          xoff[k][ax] = (a * (C::LB + 1) + b) * C::KSZ + c * (C::LD + 1) + d;
        }
      }
    }
  }
  const int ntasks = (gp.njobs + C::SLOTS - 1) / C::SLOTS;
  const int n = gp.n;

  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(counter, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int jslot = task * C::SLOTS + myslot;
    const bool have = lane_live && jslot < gp.njobs;
    int X = 0, Y = 0, Z = 0, W = 0, KX = 0, KY = 0, pbo = 0, pko = 0, nkl = 0;
    bool xs = false;
    double w = 1.0;
    if (have) {
      const GradJob jb = gp.jobs[gp.order[jslot]];
      const PairInfo pb = gp.pairs[jb.bp], pk = gp.pairs[jb.kp];
      xs = jb.xsecond != 0;
      X = xs ? pb.jsh : pb.ish;
      Y = xs ? pb.ish : pb.jsh;
      Z = pk.ish;
      W = pk.jsh;
      KX = gp.bas[8 * X + 2];
      KY = gp.bas[8 * Y + 2];
      pbo = pb.pp_off;
      pko = pk.pp_off;
      nkl = pk.npp;
      if (pb.ish == pb.jsh) w *= 0.5;
      if (pk.ish == pk.jsh) w *= 0.5;
      if (jb.bp == jb.kp) w *= 0.5;
    }
    // Gamma (or -sum_axis Gamma(a' - 2 e_axis)) for this quartet, [row][col]
    if (have) {
      const int ox = gp.aooff[X], oy = gp.aooff[Y], oz = gp.aooff[Z], ow = gp.aooff[W];
      const double *P = gp.P;
      for (int t = rho; t < C::NBRA * C::NKET; t += C::LANES) {
        const int ic = t % C::NI, jc = (t / C::NI) % C::NJ;
        const int kc = (t / C::NBRA) % C::NK, lc = t / (C::NBRA * C::NK);
        int ax_, ay_, az_;
        cart_comp_rt(C::LI, ic, ax_, ay_, az_);
        auto gam = [&](int a) {
          const int b = oy + jc, c = oz + kc, d = ow + lc;
          return 4.0 * P[(long long)a * n + b] * P[(long long)c * n + d] -
                 P[(long long)a * n + c] * P[(long long)b * n + d] -
                 P[(long long)a * n + d] * P[(long long)b * n + c];
        };
        const int bra = ic + C::NI * jc, ket = kc + C::NK * lc;
        double *g0 = Gam + (C::ROWKET ? ket * C::NBRA + bra : bra * C::NKET + ket);
        if constexpr (MODE == 0) {
          g0[0] = w * gam(ox + ic);
        } else if constexpr (MODE == 2) {
          double v = 0.0;
          if (ax_ >= 2) v -= gam(ox + cart_pos(ax_ - 2, ay_, az_));
          if (ay_ >= 2) v -= gam(ox + cart_pos(ax_, ay_ - 2, az_));
          if (az_ >= 2) v -= gam(ox + cart_pos(ax_, ay_, az_ - 2));
          g0[0] = w * v;
        } else if constexpr (MODE == 1) {   // raised: Gamma(a' - e_d)
          g0[0] = ax_ >= 1 ? w * gam(ox + cart_pos(ax_ - 1, ay_, az_)) : 0.0;
          g0[L::GAM1] = ay_ >= 1 ? w * gam(ox + cart_pos(ax_, ay_ - 1, az_)) : 0.0;
          g0[2 * L::GAM1] = az_ >= 1 ? w * gam(ox + cart_pos(ax_, ay_, az_ - 1)) : 0.0;
        } else {                            // lowered: -(a'_d + 1) Gamma(a' + e_d)
          g0[0] = -w * (ax_ + 1) * gam(ox + cart_pos(ax_ + 1, ay_, az_));
          g0[L::GAM1] = -w * (ay_ + 1) * gam(ox + cart_pos(ax_, ay_ + 1, az_));
          g0[2 * L::GAM1] = -w * (az_ + 1) * gam(ox + cart_pos(ax_, ay_, az_ + 1));
        }
      }
    }
    int kxmax = KX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) kxmax = max(kxmax, __shfl_xor_sync(0xffffffffu, kxmax, o));
    int inner = KY * nkl, innermax = inner;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) innermax = max(innermax, __shfl_xor_sync(0xffffffffu, innermax, o));
    double rA[3] = {0, 0, 0}, rB[3] = {0, 0, 0}, rC[3] = {0, 0, 0}, rD[3] = {0, 0, 0};
    if (have) {
      const int a = C::IB ? X : Y, b = C::IB ? Y : X;
      const int c = C::KB ? Z : W, d = C::KB ? W : Z;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        rA[x] = gp.centers[3 * a + x]; rB[x] = gp.centers[3 * b + x];
        rC[x] = gp.centers[3 * c + x]; rD[x] = gp.centers[3 * d + x];
      }
    }
    __syncwarp();
    const double *gamrow = Gam + (C::ROWKET ? rho * C::NBRA : rho * C::NKET);
    for (int px = 0; px < kxmax; ++px) {
      double S[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) S[c] = 0.0;
      for (int q = 0; q < innermax; ++q) {
        bool run = have && px < KX && q < inner;
        PrimPair bra, ket;
        if (run) {
          const int py = q % KY, kl = q / KY;
          const int ij = xs ? py + KY * px : px + KX * py;
          ket = gp.pp[pko + kl];
          bra = gp.pp[pbo + ij];
          run = !(ket.cce > gp.expcutoff) && !(bra.cce > gp.expcutoff - ket.cce);
        }
        double aij = 1.0, akl = 1.0, inv = 1.0, fac1 = 0.0, x = 0.0;
        double pq[3] = {0, 0, 0};
        if (run) {
          aij = bra.a; akl = ket.a;
          inv = 1.0 / (aij + akl);
          fac1 = sqrt(inv) * bra.facia * ket.facia;
          pq[0] = bra.px - ket.px; pq[1] = bra.py - ket.py; pq[2] = bra.pz - ket.pz;
          x = aij * akl * inv * (pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2]);
          for (int f = rho; f < 2 * C::NR; f += C::LANES) {
            const double v = rys_function<C::NR>(tab, x, f);
            RW[f] = v;
            if (f < C::NR) RW[2 * C::NR + f] = 1.0 / (1.0 + v);   // t^2 complement 1/(1+u)
          }
        }
        __syncwarp();
        if (run) {
          for (int u = rho; u < 3 * C::NR; u += C::LANES) {
            const int r = u / 3, ax = u - 3 * r;
            const double pa = pick3(bra.px - rA[0], bra.py - rA[1], bra.pz - rA[2], ax);
            const double qc = pick3(ket.px - rC[0], ket.py - rC[1], ket.pz - rC[2], ax);
            const double pqa = pick3(pq[0], pq[1], pq[2], ax);
            const double ab = pick3(rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2], ax);
            const double cd = pick3(rC[0] - rD[0], rC[1] - rD[1], rC[2] - rD[2], ax);
            const double d = RW[2 * C::NR + r];
            const double tmp5 = 0.5 * inv * RW[r] * d;
            const double b10 = tmp5 + 0.5 * bra.ia * d;
            const double b01 = tmp5 + 0.5 * ket.ia * d;
            const double cn = pa - 2.0 * tmp5 * akl * pqa;
            const double cm = qc + 2.0 * tmp5 * aij * pqa;
            const double v00 = ax == 2 ? RW[C::NR + r] * fac1 : 1.0;
            vrr_hrr_unit<C, double>(G + (r * 3 + ax) * C::GSZ, Tsc + u * C::TSZ, v00, cn, cm, b10,
                                    b01, tmp5, ab, cd);
          }
        }
        __syncwarp();
        if (run) {
#pragma unroll
          for (int r = 0; r < C::NR; ++r) {
            const double *gx = G + (r * 3 + 0) * C::GSZ, *gy = G + (r * 3 + 1) * C::GSZ;
            const double *gz = G + (r * 3 + 2) * C::GSZ;
            if (rho < C::NROWS) {
              double vx[C::CW], vy[C::CW], vz[C::CW];
#pragma unroll
              for (int m = 0; m < C::CW; ++m) {
                vx[m] = gx[roff[0] + m]; vy[m] = gy[roff[1] + m]; vz[m] = gz[roff[2] + m];
              }
              gout_gamma<C, NC, L::GAM1, 0>(S, gamrow, vx, vy, vz);
            }
            if constexpr (C::NEX > 0) {
#pragma unroll
              for (int k = 0; k < C::NEX; ++k)
                if (xrow[k] >= 0) {
                  const double *g = Gam + (C::ROWKET ? xrow[k] * C::NBRA + xcol[k] : xrow[k] * C::NKET + xcol[k]);
                  const double prod = gx[xoff[k][0]] * gy[xoff[k][1]] * gz[xoff[k][2]];
#pragma unroll
                  for (int c = 0; c < NC; ++c) S[c] = fma(g[c * L::GAM1], prod, S[c]);
                }
            }
          }
        }
        __syncwarp();
      }
      // reduce over the slot's lanes (extra elements live on all 32 lanes)
#pragma unroll
      for (int c = 0; c < NC; ++c) red[32 * c + rho] = 0.0;
      __syncwarp();
      double tot[NC];
      if (C::NEX > 0) {
        // one slot per warp when rows exceed 32: plain warp reduction
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double v = S[c];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          tot[c] = v;
        }
      } else {
        if (lane_live) {
#pragma unroll
          for (int c = 0; c < NC; ++c) red[32 * c + rho] = S[c];
        }
        __syncwarp();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double t = 0.0;
          for (int k = 0; k < C::LANES; ++k) t += red[32 * c + k];
          tot[c] = t;
        }
      }
      const bool writer = C::NEX > 0 ? lane == 0 : rho == 0;
      if (writer && have && px < KX) {
        if constexpr (MODE == 0 || MODE == 2) {
          const double c = gp.env[gp.bas[8 * X + 6] + px];
          const int idx = MODE == 2 ? gp.bas[8 * X + 5] + px : gp.bas[8 * X + 6] + px;
          const double val = MODE == 2 ? tot[0] : (c != 0.0 ? tot[0] / c : 0.0);
          atomicAdd(&gp.grad[idx - gp.s1], val);
        } else {
          // raised part carries 2 a_p of this primitive; lowered part none
          const double f = MODE == 1 ? 2.0 * gp.env[gp.bas[8 * X + 5] + px] : 1.0;
          double *g = gp.gatom + 3 * gp.bas[8 * X];
#pragma unroll
          for (int c = 0; c < NC; ++c) atomicAdd(&g[c], f * tot[c]);
        }
      }
      __syncwarp();
    }
    __syncwarp();
  }
}

}  // namespace lrb
