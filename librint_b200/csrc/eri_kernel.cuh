// Templated Rys ERI kernel for one canonical angular class (see
// eri_device.cuh for the decomposition).  Output mode writes every
// contracted shell quartet as a libcint block (cartesian or spherical).
#pragma once
#include "eri_device.cuh"

namespace lrb {

constexpr int ERI_WARPS = 4;                 // warps per CTA
constexpr int ERI_THREADS = 32 * ERI_WARPS;

template <int LI_, int LJ_, int LK_, int LL_>
struct EriClass {
  static constexpr int LI = LI_, LJ = LJ_, LK = LK_, LL = LL_;
  static constexpr bool IB = LI > LJ;        // bra base is i (else j)
  static constexpr bool KB = LK > LL;        // ket base is k (else l)
  static constexpr int LA = IB ? LI : LJ, LB = IB ? LJ : LI;
  static constexpr int LC = KB ? LK : LL, LD = KB ? LL : LK;
  static constexpr int NAB = LA + LB, NCD = LC + LD;
  static constexpr int NR = (LI + LJ + LK + LL) / 2 + 1;
  static constexpr int NROW = range_count(LA, NAB);   // e components
  static constexpr int NCOL = range_count(LC, NCD);   // f components
  static constexpr int SLOTS = 32 / NROW;
  static constexpr int VSZ = (NAB + 1) * (NCD + 1);
};

template <class C>
struct EriLayout {
  static constexpr int NKC = ncart(C::LK) * ncart(C::LL);   // ket (cart) columns
  // per-slot doubles: VRR tables + roots during the primitive loop; in the
  // epilogue the contracted rows F[e][f] and the half-transformed E[e][kl]
  static constexpr int LOOP = C::NR * 3 * C::VSZ + 2 * C::NR;
  static constexpr int EPI = C::NROW * (C::NCOL + NKC);
  static constexpr int SLOT = LOOP > EPI ? LOOP : EPI;
  static constexpr int WARP = C::SLOTS * SLOT;
  static constexpr int TAB = (RYS_TAB_OFFSET[C::NR + 1] - RYS_TAB_OFFSET[C::NR]);
  static constexpr size_t SMEM = sizeof(double) * (size_t)(TAB + ERI_WARPS * WARP);
};

// 2D VRR of one (root, axis) into V[n*(NCD+1)+m] (reference
// src/g2e.rs:316-506 and src/eri.rs:308-365, built on the base centres).
template <int NAB, int NCD>
__device__ __forceinline__ void vrr_2d(double *V, double v00, double cn, double cm,
                                       double b10, double b01, double b00) {
  double g[NAB + 1][NCD + 1];
  g[0][0] = v00;
#pragma unroll
  for (int m = 1; m <= NCD; ++m) {
    double v = cm * g[0][m - 1];
    if (m > 1) v = fma((m - 1) * b01, g[0][m - 2], v);
    g[0][m] = v;
  }
#pragma unroll
  for (int n = 1; n <= NAB; ++n) {
#pragma unroll
    for (int m = 0; m <= NCD; ++m) {
      double v = cn * g[n - 1][m];
      if (n > 1) v = fma((n - 1) * b10, g[n - 2][m], v);
      if (m > 0) v = fma(m * b00, g[n - 1][m - 1], v);
      g[n][m] = v;
    }
  }
#pragma unroll
  for (int n = 0; n <= NAB; ++n)
#pragma unroll
    for (int m = 0; m <= NCD; ++m) V[n * (NCD + 1) + m] = g[n][m];
}

// ---------------------------------------------------------------- epilogue
// Runtime helpers (the epilogue runs once per contracted shell quartet, so
// compact code beats full unrolling here).
__device__ __forceinline__ void cart_comp_rt(int l, int n, int &x, int &y, int &z) {
  int t = 0;
  while ((t + 1) * (t + 2) / 2 <= n) ++t;
  z = n - t * (t + 1) / 2;
  y = t - z;
  x = l - t;
}
__device__ __forceinline__ int range_index_rt(int lo, int x, int y, int z) {
  const int e = x + y + z;
  const int off = e * (e + 1) * (e + 2) / 6 - lo * (lo + 1) * (lo + 2) / 6;
  return off + (y + z) * (y + z + 1) / 2 + z;
}
__device__ __forceinline__ int binom_rt(int n, int k) {
  return k == 0 || k == n ? 1 : (n == 2 ? 2 : (n == 3 ? 3 : (n == 4 ? (k == 2 ? 6 : 4) : n)));
}
// (x-R_B)^b = sum_t C(b,t) (R_A-R_B)^(b-t) (x-R_A)^t per axis applied to a
// row of values indexed by momenta lo.. on the base centre (reference
// src/g2e.rs:507-909 applies the same shift recursively).
__device__ __forceinline__ double ipow_rt(double x, int k) {
  double r = 1.0;
  for (int i = 0; i < k; ++i) r *= x;
  return r;
}
__device__ __forceinline__ double hrr_rt(const double *src, int stride, int lo, int ax, int ay,
                                         int az, int bx, int by, int bz, double dx, double dy,
                                         double dz) {
  double s = 0.0;
  for (int tx = 0; tx <= bx; ++tx)
    for (int ty = 0; ty <= by; ++ty)
      for (int tz = 0; tz <= bz; ++tz) {
        const double c = (double)(binom_rt(bx, tx) * binom_rt(by, ty) * binom_rt(bz, tz)) *
                         ipow_rt(dx, bx - tx) * ipow_rt(dy, by - ty) * ipow_rt(dz, bz - tz);
        s = fma(c, src[stride * range_index_rt(lo, ax + tx, ay + ty, az + tz)], s);
      }
  return s;
}

// cart->sph coefficients, c2s[l][m][c] for l <= 4 (filled by the host from
// the real-solid-harmonic closed form; libcint order and normalisation).
constexpr int C2S_L = 5, C2S_M = 9, C2S_C = 15;
// One copy per translation unit (no relocatable device code); each unit's
// class-registration function uploads it.
static __constant__ double c_c2s[C2S_L * C2S_M * C2S_C];
__device__ __forceinline__ double c2s(int l, int m, int c) { return c_c2s[(l * C2S_M + m) * C2S_C + c]; }

// Persistent kernel: warps pull tasks (SLOTS quartets each) from *counter.
template <int LI, int LJ, int LK, int LL>
__global__ void __launch_bounds__(ERI_THREADS)
k_eri_out(EriParams prm, const double *__restrict__ rys_tab_n, int *counter) {
  using C = EriClass<LI, LJ, LK, LL>;
  using L = EriLayout<C>;
  extern __shared__ double smem[];
  double *tab = smem;
  // stage this class's root table (same for every CTA)
  for (int i = threadIdx.x; i < L::TAB; i += blockDim.x) tab[i] = rys_tab_n[i];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *wbuf = smem + L::TAB + warp * L::WARP;
  const int slot = lane / C::NROW;
  const int rho = lane - slot * C::NROW;
  const bool lane_live = slot < C::SLOTS;
  const int myslot = lane_live ? slot : C::SLOTS - 1;
  double *sb = wbuf + myslot * L::SLOT;        // this slot's area
  double *Vs = sb;                             // [NR][3][VSZ]
  double *RW = sb + C::NR * 3 * C::VSZ;        // [2*NR]
  // row components of this lane
  int ex = 0, ey = 0, ez = 0;
  {
    int r = rho < C::NROW ? rho : 0, e = C::LA;
    while (r >= ncart(e)) { r -= ncart(e); ++e; }
    cart_comp_rt(e, r, ex, ey, ez);
  }
  const bool sph = prm.sph != 0;
  constexpr int NI = ncart(LI), NJ = ncart(LJ), NK = ncart(LK), NL = ncart(LL);
  const int NIo = sph ? nsph(LI) : NI, NJo = sph ? nsph(LJ) : NJ;
  const int NKo = sph ? nsph(LK) : NK, NLo = sph ? nsph(LL) : NL;
  const int NKO = NKo * NLo, NBO = NIo * NJo;
  const int ntasks = (prm.njobs + C::SLOTS - 1) / C::SLOTS;

  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(counter, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int jslot = task * C::SLOTS + myslot;
    const bool have = lane_live && jslot < prm.njobs;
    QuartetJob job;
    if (have) job = prm.jobs[prm.order[jslot]];
    else { job.nij = 0; job.nkl = 0; job.pij_off = job.pkl_off = 0; }
    const int np = job.nij * job.nkl;
    int npmax = np;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) npmax = max(npmax, __shfl_xor_sync(0xffffffffu, npmax, o));

    // centres: A/B on the bra, C/D on the ket
    double rA[3] = {0, 0, 0}, rB[3] = {0, 0, 0}, rC[3] = {0, 0, 0}, rD[3] = {0, 0, 0};
    if (have) {
      const int a = C::IB ? job.ish : job.jsh, b = C::IB ? job.jsh : job.ish;
      const int c = C::KB ? job.ksh : job.lsh, d = C::KB ? job.lsh : job.ksh;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        rA[x] = prm.centers[3 * a + x]; rB[x] = prm.centers[3 * b + x];
        rC[x] = prm.centers[3 * c + x]; rD[x] = prm.centers[3 * d + x];
      }
    }
    double acc[C::NCOL];
#pragma unroll
    for (int c = 0; c < C::NCOL; ++c) acc[c] = 0.0;

    int ij = 0, kl = 0;
    for (int p = 0; p < npmax; ++p) {
      bool run = p < np;
      PrimPair bra, ket;
      if (run) {
        ket = prm.pp[job.pkl_off + kl];
        bra = prm.pp[job.pij_off + ij];
        // screening (reference src/cint2e.rs:367-393)
        run = !(ket.cce > prm.expcutoff) && !(bra.cce > prm.expcutoff - ket.cce);
      }
      if (++ij == job.nij) { ij = 0; ++kl; }
      double aij = 1.0, akl = 1.0, a0 = 1.0, fac1 = 0.0, x = 0.0;
      double pq[3] = {0, 0, 0};
      if (run) {
        aij = bra.a; akl = ket.a;
        const double a1 = aij * akl;
        a0 = a1 / (aij + akl);
        fac1 = sqrt(a0 / (a1 * a1 * a1)) * bra.fac * ket.fac;
        pq[0] = bra.px - ket.px; pq[1] = bra.py - ket.py; pq[2] = bra.pz - ket.pz;
        x = a0 * (pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2]);
        for (int f = rho; f < 2 * C::NR; f += C::NROW) RW[f] = rys_function<C::NR>(tab, x, f);
      }
      __syncwarp();
      if (run) {
        const double pa[3] = {bra.px - rA[0], bra.py - rA[1], bra.pz - rA[2]};
        const double qc[3] = {ket.px - rC[0], ket.py - rC[1], ket.pz - rC[2]};
        for (int u = rho; u < 3 * C::NR; u += C::NROW) {
          const int r = u / 3, ax = u - 3 * r;
          const double u2 = a0 * RW[r];
          const double tmp4 = 0.5 / (u2 * (aij + akl) + aij * akl);
          const double tmp5 = u2 * tmp4;
          const double b10 = tmp5 + tmp4 * akl;
          const double b01 = tmp5 + tmp4 * aij;
          const double cn = pa[ax] - 2.0 * tmp5 * akl * pq[ax];
          const double cm = qc[ax] + 2.0 * tmp5 * aij * pq[ax];
          const double v00 = ax == 2 ? RW[C::NR + r] * fac1 : 1.0;
          vrr_2d<C::NAB, C::NCD>(Vs + (r * 3 + ax) * C::VSZ, v00, cn, cm, b10, b01, tmp5);
        }
      }
      __syncwarp();
      if (run && rho < C::NROW) {
#pragma unroll
        for (int r = 0; r < C::NR; ++r) {
          const double *vxp = Vs + (r * 3 + 0) * C::VSZ + ex * (C::NCD + 1);
          const double *vyp = Vs + (r * 3 + 1) * C::VSZ + ey * (C::NCD + 1);
          const double *vzp = Vs + (r * 3 + 2) * C::VSZ + ez * (C::NCD + 1);
          double vx[C::NCD + 1], vy[C::NCD + 1], vz[C::NCD + 1];
#pragma unroll
          for (int m = 0; m <= C::NCD; ++m) { vx[m] = vxp[m]; vy[m] = vyp[m]; vz[m] = vzp[m]; }
#pragma unroll
          for (int c = 0; c < C::NCOL; ++c)
            acc[c] = fma(vx[range_x(C::LC, c)] * vy[range_y(C::LC, c)], vz[range_z(C::LC, c)], acc[c]);
        }
      }
      __syncwarp();
    }

    // ---------------------------------------------------------- epilogue
    // HRR after contraction, then cart->sph, per shell quartet.
    const double cdx = rC[0] - rD[0], cdy = rC[1] - rD[1], cdz = rC[2] - rD[2];
    const double abx = rA[0] - rB[0], aby = rA[1] - rB[1], abz = rA[2] - rB[2];
    double *F = sb;                            // [NROW][NCOL]
    double *E = sb + C::NROW * C::NCOL;        // [NROW][NKO]
    if (have && rho < C::NROW) {
#pragma unroll
      for (int c = 0; c < C::NCOL; ++c) F[rho * C::NCOL + c] = acc[c];
    }
    __syncwarp();
    if (have) {
      // ket: [e|f] -> [e|kl] in output (k fastest) order
      for (int t = rho; t < C::NROW * NKO; t += C::NROW) {
        const int e = t / NKO, kap = t - e * NKO;
        const int ko = kap % NKo, lo = kap / NKo;
        double v = 0.0;
        for (int kc = 0; kc < NK; ++kc) {
          const double ck = sph ? c2s(LK, ko, kc) : (kc == ko ? 1.0 : 0.0);
          if (ck == 0.0) continue;
          int kx, ky, kz;
          cart_comp_rt(LK, kc, kx, ky, kz);
          for (int lc = 0; lc < NL; ++lc) {
            const double cl = sph ? c2s(LL, lo, lc) : (lc == lo ? 1.0 : 0.0);
            if (cl == 0.0) continue;
            int lx, ly, lz;
            cart_comp_rt(LL, lc, lx, ly, lz);
            const double h = C::KB ? hrr_rt(F + e * C::NCOL, 1, C::LC, kx, ky, kz, lx, ly, lz, cdx, cdy, cdz)
                                   : hrr_rt(F + e * C::NCOL, 1, C::LC, lx, ly, lz, kx, ky, kz, cdx, cdy, cdz);
            v = fma(ck * cl, h, v);
          }
        }
        E[t] = v;
      }
    }
    __syncwarp();
    if (have) {
      // bra: [e|kl] -> (ij|kl), written to global (i fastest -> coalesced)
      for (int t = rho; t < NKO * NBO; t += C::NROW) {
        const int kap = t / NBO, b = t - kap * NBO;
        const int io = b % NIo, jo = b / NIo;
        const int ko = kap % NKo, lo = kap / NKo;
        double v = 0.0;
        for (int ic = 0; ic < NI; ++ic) {
          const double ci = sph ? c2s(LI, io, ic) : (ic == io ? 1.0 : 0.0);
          if (ci == 0.0) continue;
          int ix, iy, iz;
          cart_comp_rt(LI, ic, ix, iy, iz);
          for (int jc = 0; jc < NJ; ++jc) {
            const double cj = sph ? c2s(LJ, jo, jc) : (jc == jo ? 1.0 : 0.0);
            if (cj == 0.0) continue;
            int jx, jy, jz;
            cart_comp_rt(LJ, jc, jx, jy, jz);
            const double h = C::IB ? hrr_rt(E + kap, NKO, C::LA, ix, iy, iz, jx, jy, jz, abx, aby, abz)
                                   : hrr_rt(E + kap, NKO, C::LA, jx, jy, jz, ix, iy, iz, abx, aby, abz);
            v = fma(ci * cj, h, v);
          }
        }
        prm.out[job.out_off + (long long)io * job.s_i + (long long)jo * job.s_j +
                (long long)ko * job.s_k + (long long)lo * job.s_l] = v;
      }
    }
    __syncwarp();
  }
}

}  // namespace lrb
