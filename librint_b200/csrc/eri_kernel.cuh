// Templated Rys ERI kernel for one canonical angular class (LI LJ | LK LL),
// LI >= LJ, LK >= LL, (LI,LJ) >= (LK,LL).
//
// Per primitive quartet and Rys root (reference src/g2e.rs:5539-5679 and
// src/eri.rs:263-399):
//   * roots/weights u_r, w_r from the piecewise tables staged in shared
//     memory (one lane per node or weight);
//   * one lane per (root, axis) builds the 2D table V(n, m) on the base
//     centres A (bra) and C (ket) -- i if LI > LJ else j, k if LK > LL else
//     l, as src/g2e.rs:113-181 chooses -- then shifts it to the partners by
//     the horizontal recurrences on these 1D arrays, giving G[a][b][c][d];
//   * gout: every lane owns one row of the final cartesian block (the smaller
//     of the bra/ket sides, but the bra of (dd|ps), (dd|pp), (dd|dp)) and
//     accumulates all columns in registers:
//     I(row, col) += Gx Gy Gz (src/cint2e.rs:2456-2895).
// The recurrences stay per primitive (as the reference does) because shifting
// after contraction acts on 3D products and loses ~2 digits for distant
// centres.  A warp holds SLOTS = 32 / rows quartets; rows beyond 32 ((dd|dd))
// are split across lanes by columns.  The epilogue transforms to spherical
// harmonics and writes libcint blocks (MODE 0) or digests the cartesian block
// into J/K (MODE 1).
#pragma once
#include "eri_device.cuh"

namespace lrb {

constexpr int ERI_WARPS = 4;                 // warps per CTA
constexpr int ERI_THREADS = 32 * ERI_WARPS;

template <int LI_, int LJ_, int LK_, int LL_, bool PACK = false>
struct EriClass {
  static constexpr int LI = LI_, LJ = LJ_, LK = LK_, LL = LL_;
  static constexpr bool IB = LI > LJ;        // bra base is i (else j)
  static constexpr bool KB = LK > LL;        // ket base is k (else l)
  static constexpr int LA = IB ? LI : LJ, LB = IB ? LJ : LI;
  static constexpr int LC = KB ? LK : LL, LD = KB ? LL : LK;
  static constexpr int NAB = LA + LB, NCD = LC + LD;
  static constexpr int NR = (LI + LJ + LK + LL) / 2 + 1;
  static constexpr int NI = ncart(LI), NJ = ncart(LJ), NK = ncart(LK), NL = ncart(LL);
  static constexpr int NBRA = NI * NJ, NKET = NK * NL;
  // Rows are the smaller side, except (dd|ps), (dd|pp) and (dd|dp) of the
  // ERI / Fock kernels (PACK), which run 36 bra rows (32 lanes plus split
  // extras) against ket columns: measured on the K = 1..6 sweep, 17 %, 38 %
  // and 4.5 % faster than 3, 9 or 18 ket rows (fewer accumulators per lane,
  // one round of (root, axis) units over 32 lanes).
  static constexpr bool BRA_ROWS =
      PACK && LI_ == 2 && LJ_ == 2 && ((LK_ == 1 && LL_ <= 1) || (LK_ == 2 && LL_ == 1));
  static constexpr bool ROWKET = !BRA_ROWS && NKET <= NBRA;   // rows are ket components
  static constexpr int NROWS = ROWKET ? NKET : NBRA;
  static constexpr int NCOLS = ROWKET ? NBRA : NKET;
  // Lanes per slot.  Each of the LANES lanes owns one row; rows beyond LANES
  // are split by columns over the slot's lanes ("extra" elements).  With
  // PACK the count is chosen by a cost model of one primitive iteration: a
  // round of (root, axis) units costs ~350 instruction slots, a row column
  // ~2.75 per root and an extra element twice that; 18-row classes then run
  // two 16-lane slots per warp instead of one 18-lane slot.
  static constexpr double lane_rate(int L) {
    const int ex = NROWS > L ? ((NROWS - L) * NCOLS + L - 1) / L : 0;
    const int units = (3 * NR + L - 1) / L;
    return (32 / L) / (units * 350.0 + NR * (NCOLS + 2.0 * ex) * 2.75);
  }
  static constexpr int pick_lanes() {
    if (NROWS >= 32 || !PACK) return NROWS < 32 ? NROWS : 32;
    int best = NROWS;
    double rate = lane_rate(NROWS);
    // at most 5 extra elements per lane (their offsets live in registers)
    // and at most 88 KB of slot memory per CTA (with the root table, two CTAs per SM)
    for (int L = 16; L >= 8; L /= 2)
      if (L < NROWS && ((NROWS - L) * NCOLS + L - 1) / L <= 5 &&
          ERI_WARPS * (32 / L) * slot_doubles() * 8 <= 88 * 1024 && lane_rate(L) > 1.05 * rate) {
        best = L;
        rate = lane_rate(L);
      }
    return best;
  }
  static constexpr int LANES = pick_lanes();
  static constexpr int SLOTS = 32 / LANES;
  static constexpr int EXTRA = NROWS > LANES ? (NROWS - LANES) * NCOLS : 0;   // split elements
  static constexpr int NEX = (EXTRA + LANES - 1) / LANES;                      // per lane
  // G[a][b][c][d] sizes; row-side indices first, column side contiguous
  static constexpr int BSZ = (LA + 1) * (LB + 1), KSZ = (LC + 1) * (LD + 1);
  static constexpr int GSZ = BSZ * KSZ;
  static constexpr int CW = ROWKET ? BSZ : KSZ;   // column values per axis
  // after the bra shift; not needed when the ket has no shift (LD == 0)
  static constexpr int TSZ = LD > 0 ? BSZ * (NCD + 1) : 0;
  // shared-memory strides of the per-(root, axis) G arrays and bra-shift
  // scratch, odd so that the units' lanes, which write and read their own
  // arrays in step, fall on distinct banks (an even stride put lanes 2k and
  // 2k + 16 words apart on the same banks)
  static constexpr int GST = GSZ | 1;
  static constexpr int TST = TSZ > 0 ? (TSZ | 1) : 0;
  // shared-memory doubles of one slot (loop area or output epilogue)
  static constexpr int slot_doubles() {
    const int loop = 3 * NR + 3 * NR * GST + 3 * NR * TST;
    const int epi = 2 * NBRA * NKET;
    return loop > epi ? loop : epi;
  }

  // component c of cartesian function n of momentum l
  static constexpr int cc(int l, int n, int axis) {
    return axis == 0 ? cart_x(l, n) : (axis == 1 ? cart_y(l, n) : cart_z(l, n));
  }
  // bra (ic, jc) -> offset of (a, b) in a BSZ block for one axis
  static constexpr int bra_off(int ic, int jc, int axis) {
    return IB ? cc(LI, ic, axis) * (LB + 1) + cc(LJ, jc, axis)
              : cc(LJ, jc, axis) * (LB + 1) + cc(LI, ic, axis);
  }
  static constexpr int ket_off(int kc, int lc, int axis) {
    return KB ? cc(LK, kc, axis) * (LD + 1) + cc(LL, lc, axis)
              : cc(LL, lc, axis) * (LD + 1) + cc(LK, kc, axis);
  }
  // column k (compile time) -> offset inside a row's CW values, per axis
  static constexpr int col_off(int k, int axis) {
    return ROWKET ? bra_off(k % NI, k / NI, axis) : ket_off(k % NK, k / NK, axis);
  }
};

// Density sub-blocks a quartet's digestion reads, staged once per quartet in
// the slot's shared memory (the digestion reads each of them NI..NL times):
// P_cd, P_ab, P_bd, P_ad, P_bc, P_ac, each row-major in (first, second).
template <int NI, int NJ, int NK, int NL>
struct FockStage {
  static constexpr int CD = 0, AB = CD + NK * NL, BD = AB + NI * NJ, AD = BD + NJ * NL,
                       BC = AD + NI * NL, AC = BC + NJ * NK, SIZE = AC + NI * NK;
};

template <class C, int MODE = 0, typename R = double>
struct EriLayout {
  static constexpr int NKO_MAX = C::NKET;   // cartesian >= spherical
  // per-slot sizes in doubles: roots, weights, 1/(1+u) (3 NR, FP64), then G
  // (NR*3*GST) and per-unit bra-shift scratch (3*NR*TST) in the arithmetic
  // type R in the loop; block (NBRA*NKET, R) + ket-transformed block
  // (NBRA*NKO, output mode only) in the epilogue.  FP32 halves the R parts.
  static constexpr int RD(int n) { return (int)((n * sizeof(R) + 7) / 8); }
  static constexpr int LOOP = 3 * C::NR + RD(C::NR * 3 * C::GST + C::NR * 3 * C::TST);
  // Fock mode stages the quartet's density blocks after the block
  static constexpr int EPI = RD(C::NBRA * C::NKET) +
                             (MODE == 0 ? C::NBRA * NKO_MAX
                                        : RD(FockStage<C::NI, C::NJ, C::NK, C::NL>::SIZE) + 1);
  // odd, so that 1-lane slots (32 per warp, each lane in its own slot) put
  // the lanes' same-offset accesses on distinct banks
  static constexpr int SLOT = (LOOP > EPI ? LOOP : EPI) | 1;
  static constexpr int WARP = C::SLOTS * SLOT;
  static constexpr int TAB = (RYS_TAB_OFFSET[C::NR + 1] - RYS_TAB_OFFSET[C::NR]);
  static constexpr int C2S = 3 * 5 * 6;    // l <= 2, m, cart
  static constexpr size_t SMEM = sizeof(double) * (size_t)(TAB + C2S + ERI_WARPS * WARP);
};

// cart->sph coefficients, c2s[l][m][c] for l <= 4 (filled by the host from
// the real-solid-harmonic closed form; libcint order and normalisation).
// One copy per translation unit; each unit's registration uploads it.
constexpr int C2S_L = 5, C2S_M = 9, C2S_C = 15;
static __constant__ double c_c2s[C2S_L * C2S_M * C2S_C];

// ---------------------------------------------------------------- unit
// One (root, axis): 2D VRR on (A, C), bra shift A->B for every m, ket shift
// C->D, result G[row side][column side] written to shared memory.
template <class C, typename R>
__device__ __forceinline__ void vrr_hrr_unit(R *G, R *T, R v00, R cn, R cm, R b10, R b01, R b00,
                                             R ab, R cd) {
  constexpr int NAB = C::NAB, NCD = C::NCD, LA = C::LA, LB = C::LB, LC = C::LC, LD = C::LD;
  R g[NAB + 1][NCD + 1];
  g[0][0] = v00;
#pragma unroll
  for (int m = 1; m <= NCD; ++m) {
    R v = cm * g[0][m - 1];
    if (m > 1) v = fma(R(m - 1) * b01, g[0][m - 2], v);
    g[0][m] = v;
  }
#pragma unroll
  for (int n = 1; n <= NAB; ++n)
#pragma unroll
    for (int m = 0; m <= NCD; ++m) {
      R v = cn * g[n - 1][m];
      if (n > 1) v = fma(R(n - 1) * b10, g[n - 2][m], v);
      if (m > 0) v = fma(R(m) * b00, g[n - 1][m - 1], v);
      g[n][m] = v;
    }
  // bra shift per m column: h[a][b] from g[a+b'][m], (x-B) = (x-A) + (A-B)
#pragma unroll
  for (int m = 0; m <= NCD; ++m) {
    R h[NAB + 1][LB + 1];
#pragma unroll
    for (int n = 0; n <= NAB; ++n) h[n][0] = g[n][m];
#pragma unroll
    for (int b = 1; b <= LB; ++b)
#pragma unroll
      for (int a = 0; a <= NAB - b; ++a) h[a][b] = fma(ab, h[a][b - 1], h[a + 1][b - 1]);
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
      for (int b = 0; b <= LB; ++b) {
        if constexpr (LD == 0) {   // no ket shift: m is the ket index c
          const int bi = a * (LB + 1) + b;
          G[C::ROWKET ? m * C::BSZ + bi : bi * C::KSZ + m] = h[a][b];
        } else {
          T[(a * (LB + 1) + b) * (NCD + 1) + m] = h[a][b];
        }
      }
  }
  if constexpr (LD == 0) return;
  // ket shift per (a, b): k[c][d] from T[a][b][c+d']
#pragma unroll
  for (int a = 0; a <= LA; ++a)
#pragma unroll
    for (int b = 0; b <= LB; ++b) {
      R k[NCD + 1][LD + 1];
#pragma unroll
      for (int m = 0; m <= NCD; ++m) k[m][0] = T[(a * (LB + 1) + b) * (NCD + 1) + m];
#pragma unroll
      for (int d = 1; d <= LD; ++d)
#pragma unroll
        for (int c = 0; c <= NCD - d; ++c) k[c][d] = fma(cd, k[c][d - 1], k[c + 1][d - 1]);
#pragma unroll
      for (int c = 0; c <= LC; ++c)
#pragma unroll
        for (int d = 0; d <= LD; ++d) {
          const int bi = a * (LB + 1) + b, ki = c * (LD + 1) + d;
          G[C::ROWKET ? ki * C::BSZ + bi : bi * C::KSZ + ki] = k[c][d];
        }
    }
}

// acc[k] += x[col_x(k)] y[col_y(k)] z[col_z(k)] for all columns (compile-time
// offsets by recursion).
template <class C, typename R, int K>
__device__ __forceinline__ void gout_cols(R (&acc)[C::NCOLS], const R (&x)[C::CW],
                                          const R (&y)[C::CW], const R (&z)[C::CW]) {
  if constexpr (K < C::NCOLS) {
    constexpr int X = C::col_off(K, 0), Y = C::col_off(K, 1), Z = C::col_off(K, 2);
    acc[K] = fma(x[X] * y[Y], z[Z], acc[K]);
    gout_cols<C, R, K + 1>(acc, x, y, z);
  }
}

// doubles needed for `bytes` bytes
__host__ __device__ constexpr int RD_(size_t bytes) { return (int)((bytes + 7) / 8); }

// ---------------------------------------------------------------- digestion
template <int NI, int NJ, int NK, int NL, typename R>
__device__ __forceinline__ void fock_stage(R *Ps, const QuartetJob &q, const FockParams &fk,
                                           int rho, int nlanes) {
  using S = FockStage<NI, NJ, NK, NL>;
  const int n = fk.n;
  const int oi = fk.aooff[q.ish], oj = fk.aooff[q.jsh], ok = fk.aooff[q.ksh], ol = fk.aooff[q.lsh];
  const double *P = fk.P;
  for (int t = rho; t < S::SIZE; t += nlanes) {
    int r0, c0, nc, e;
    if (t < S::AB) { e = t - S::CD; r0 = ok; c0 = ol; nc = NL; }
    else if (t < S::BD) { e = t - S::AB; r0 = oi; c0 = oj; nc = NJ; }
    else if (t < S::AD) { e = t - S::BD; r0 = oj; c0 = ol; nc = NL; }
    else if (t < S::BC) { e = t - S::AD; r0 = oi; c0 = ol; nc = NL; }
    else if (t < S::AC) { e = t - S::BC; r0 = oj; c0 = ok; nc = NK; }
    else { e = t - S::AC; r0 = oi; c0 = ok; nc = NK; }
    Ps[t] = (R)P[(long long)(r0 + e / nc) * n + c0 + e % nc];
  }
}

// J/K digestion of one cartesian block B[a + NI*(b + NJ*(c + NK*d))] with
// the degeneracy weight w of its canonical shell quartet, against the staged
// density blocks Ps:
//   Jacc[ab] += 2w sum_cd B P[cd],  Jacc[cd] += 2w sum_ab B P[ab],
//   Kacc[ac] += w sum_bd B P[bd],   Kacc[bc] += w sum_ad B P[ad],
//   Kacc[ad] += w sum_bc B P[bc],   Kacc[bd] += w sum_ac B P[ac];
// G = (Jacc + Jacc^T) - (Kacc + Kacc^T)/2 then equals the reference's
// G[mu nu] = sum P[ls](mu nu|s l) - 1/2 sum P[ns](mu l|s n) (src/scf.rs:379-391).
template <int NI, int NJ, int NK, int NL, typename R>
__device__ __forceinline__ void fock_digest(const R *B, const R *Ps, const QuartetJob &q, double w,
                                            const FockParams &fk, int rho, int nlanes) {
  using S = FockStage<NI, NJ, NK, NL>;
  const int n = fk.n;
  const int oi = fk.aooff[q.ish], oj = fk.aooff[q.jsh], ok = fk.aooff[q.ksh], ol = fk.aooff[q.lsh];
  auto blk = [&](int a, int b, int c, int d) { return B[a + NI * (b + NJ * (c + NK * d))]; };
  for (int t = rho; t < NI * NJ; t += nlanes) {          // J[ab]
    const int a = t % NI, b = t / NI;
    R s = 0;
    for (int d = 0; d < NL; ++d)
      for (int c = 0; c < NK; ++c) s = fma(blk(a, b, c, d), Ps[S::CD + c * NL + d], s);
    atomicAdd(&fk.J[(long long)(oi + a) * n + oj + b], 2.0 * w * (double)s);
  }
  for (int t = rho; t < NK * NL; t += nlanes) {          // J[cd]
    const int c = t % NK, d = t / NK;
    R s = 0;
    for (int b = 0; b < NJ; ++b)
      for (int a = 0; a < NI; ++a) s = fma(blk(a, b, c, d), Ps[S::AB + a * NJ + b], s);
    atomicAdd(&fk.J[(long long)(ok + c) * n + ol + d], 2.0 * w * (double)s);
  }
  for (int t = rho; t < NI * NK; t += nlanes) {          // K[ac]
    const int a = t % NI, c = t / NI;
    R s = 0;
    for (int d = 0; d < NL; ++d)
      for (int b = 0; b < NJ; ++b) s = fma(blk(a, b, c, d), Ps[S::BD + b * NL + d], s);
    atomicAdd(&fk.K[(long long)(oi + a) * n + ok + c], w * (double)s);
  }
  for (int t = rho; t < NJ * NK; t += nlanes) {          // K[bc]
    const int b = t % NJ, c = t / NJ;
    R s = 0;
    for (int d = 0; d < NL; ++d)
      for (int a = 0; a < NI; ++a) s = fma(blk(a, b, c, d), Ps[S::AD + a * NL + d], s);
    atomicAdd(&fk.K[(long long)(oj + b) * n + ok + c], w * (double)s);
  }
  for (int t = rho; t < NI * NL; t += nlanes) {          // K[ad]
    const int a = t % NI, d = t / NI;
    R s = 0;
    for (int c = 0; c < NK; ++c)
      for (int b = 0; b < NJ; ++b) s = fma(blk(a, b, c, d), Ps[S::BC + b * NK + c], s);
    atomicAdd(&fk.K[(long long)(oi + a) * n + ol + d], w * (double)s);
  }
  for (int t = rho; t < NJ * NL; t += nlanes) {          // K[bd]
    const int b = t % NJ, d = t / NJ;
    R s = 0;
    for (int c = 0; c < NK; ++c)
      for (int a = 0; a < NI; ++a) s = fma(blk(a, b, c, d), Ps[S::AC + a * NK + c], s);
    atomicAdd(&fk.K[(long long)(oj + b) * n + ol + d], w * (double)s);
  }
}

__device__ __forceinline__ void cart_comp_rt(int l, int n, int &x, int &y, int &z) {
  int t = 0;
  while ((t + 1) * (t + 2) / 2 <= n) ++t;
  z = n - t * (t + 1) / 2;
  y = t - z;
  x = l - t;
}

// ---------------------------------------------------------------- kernel
// Persistent: warps pull tasks (SLOTS quartets each) from *counter.
// MODE 0 writes libcint blocks; MODE 1 digests each block into J/K.
// R is the arithmetic type of the recurrences, the products and the
// digestion (double, or float for the mixed-precision Fock build); roots,
// weights and pair data are always evaluated in FP64 and rounded after.
template <int LI, int LJ, int LK, int LL, int MODE, typename R = double>
__global__ void __launch_bounds__(ERI_THREADS)
k_eri(EriParams prm, FockParams fk, const double *__restrict__ rys_tab_n, int *counter) {
  using C = EriClass<LI, LJ, LK, LL, true>;
  using L = EriLayout<C, MODE, R>;
  static_assert(MODE == 1 || sizeof(R) == 8, "output mode is FP64");
  extern __shared__ double smem[];
  double *tab = smem;
  double *c2s_s = smem + L::TAB;            // [3][5][6]
  for (int i = threadIdx.x; i < L::TAB; i += blockDim.x) tab[i] = rys_tab_n[i];
  for (int i = threadIdx.x; i < L::C2S; i += blockDim.x) {
    const int l = i / 30, m = (i / 6) % 5, c = i % 6;
    c2s_s[i] = c_c2s[(l * C2S_M + m) * C2S_C + c];
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *wbuf = smem + L::TAB + L::C2S + warp * L::WARP;
  const int slot = lane / C::LANES;
  const int rho = lane - slot * C::LANES;
  const bool lane_live = slot < C::SLOTS;
  const int myslot = lane_live ? slot : C::SLOTS - 1;
  double *sb = wbuf + myslot * L::SLOT;        // this slot's area
  double *RW = sb;                             // [3*NR] FP64 roots, weights, 1/(1+u)
  R *G = reinterpret_cast<R *>(sb + 3 * C::NR);            // [NR][3][GST]
  R *Tsc = G + C::NR * 3 * C::GST;                         // [3*NR][TST]

  // row offsets of this lane (row side indices, per axis)
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
      if (C::ROWKET) {   // row = (kc, lc) -> (c, d)
        const int c = C::KB ? pc[ax] : qc[ax], d = C::KB ? qc[ax] : pc[ax];
        roff[ax] = (c * (C::LD + 1) + d) * C::BSZ;
      } else {           // row = (ic, jc) -> (a, b)
        const int a = C::IB ? pc[ax] : qc[ax], b = C::IB ? qc[ax] : pc[ax];
        roff[ax] = (a * (C::LB + 1) + b) * C::KSZ;
      }
    }
  }
  // extra elements (rows >= 32, column split): row and column offsets
  int xrow[C::NEX > 0 ? C::NEX : 1], xoff[C::NEX > 0 ? C::NEX : 1][3];
  if constexpr (C::NEX > 0) {
#pragma unroll
    for (int k = 0; k < C::NEX; ++k) {
      const int e = rho + C::LANES * k;
      xrow[k] = e < C::EXTRA ? C::LANES + e / C::NCOLS : -1;
      const int col = e < C::EXTRA ? e % C::NCOLS : 0;
      const int row = e < C::EXTRA ? C::LANES + e / C::NCOLS : 0;
      const int p = C::ROWKET ? C::NK : C::NI;
      const int lp = C::ROWKET ? C::LK : C::LI, lq = C::ROWKET ? C::LL : C::LJ;
      const int cp = C::ROWKET ? C::NI : C::NK;
      const int lcp = C::ROWKET ? C::LI : C::LK, lcq = C::ROWKET ? C::LJ : C::LL;
      int px, py, pz, qx, qy, qz, ux, uy, uz, vx, vy, vz;
      cart_comp_rt(lp, row % p, px, py, pz);
      cart_comp_rt(lq, row / p, qx, qy, qz);
      cart_comp_rt(lcp, col % cp, ux, uy, uz);
      cart_comp_rt(lcq, col / cp, vx, vy, vz);
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
  const bool sph = MODE == 0 && prm.sph != 0;
  const int NIo = sph ? nsph(LI) : C::NI, NJo = sph ? nsph(LJ) : C::NJ;
  const int NKo = sph ? nsph(LK) : C::NK, NLo = sph ? nsph(LL) : C::NL;
  const int NKO = NKo * NLo, NBO = NIo * NJo;
  const int ntasks = (prm.njobs + C::SLOTS - 1) / C::SLOTS;
  unsigned long long nprim = 0;   // MODE 1, measurement: primitive quartets run

  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(counter, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int jslot = task * C::SLOTS + myslot;
    const bool have = lane_live && jslot < prm.njobs;
    QuartetJob job;
    double wdeg = 1.0;   // Fock mode: 1/2 per coinciding shell / pair
    if (!have) {
      job.nij = 0; job.nkl = 0; job.pij_off = job.pkl_off = 0;
    } else if (MODE == 0) {
      job = prm.jobs[prm.order[jslot]];
    } else {
      const int2 jb = fk.jobs[prm.order[jslot]];
      const PairInfo pb = fk.pairs[jb.x], pk = fk.pairs[jb.y];
      job.ish = pb.ish; job.jsh = pb.jsh; job.pij_off = pb.pp_off; job.nij = pb.npp;
      job.ksh = pk.ish; job.lsh = pk.jsh; job.pkl_off = pk.pp_off; job.nkl = pk.npp;
      job.out_off = 0; job.s_i = job.s_j = job.s_k = job.s_l = 0;
      if (pb.ish == pb.jsh) wdeg *= 0.5;
      if (pk.ish == pk.jsh) wdeg *= 0.5;
      if (jb.x == jb.y) wdeg *= 0.5;
    }
    // Primitive quartets to visit.  Output mode: each shell pair's primitive
    // pairs are sorted by ascending screening key cce, so for ket pair kl the
    // bra pairs that pass (bra.cce <= cutoff - ket.cce) are a prefix of
    // length nb(kl), non-increasing in kl; only those are visited.  Fock mode
    // keeps the pairs in natural order and tests each quartet: a cce-sorted
    // walk adds the largest contributions to the FP32 accumulators first and
    // was measured to raise the FP32 G error 3.5x, at no gain in time.
    const double cut = prm.expcutoff;
    int np = 0;
    if constexpr (MODE == 0) {
      int nb = job.nij;
      for (int k = 0; k < job.nkl; ++k) {
        const double kc = prm.pp[job.pkl_off + k].cce;
        if (!(kc <= cut)) break;
        while (nb > 0 && !(prm.pp[job.pij_off + nb - 1].cce <= cut - kc)) --nb;
        if (nb == 0) break;
        np += nb;
      }
    } else {
      np = job.nij * job.nkl;
    }
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
    R acc[C::NCOLS];
#pragma unroll
    for (int c = 0; c < C::NCOLS; ++c) acc[c] = 0;
    R xacc[C::NEX > 0 ? C::NEX : 1];
#pragma unroll
    for (int k = 0; k < (C::NEX > 0 ? C::NEX : 1); ++k) xacc[k] = 0;

    int ij = 0, kl = 0;
    int nbk = job.nij;   // output mode: passing bra prefix of the current ket pair
    if constexpr (MODE == 0) {
      if (np > 0) {
        const double kc = prm.pp[job.pkl_off].cce;
        while (nbk > 0 && !(prm.pp[job.pij_off + nbk - 1].cce <= cut - kc)) --nbk;
      }
    }
    // Range separation (omega = env[8], reference src/g2e.rs:5564-5612):
    // omega > 0 (long range, erf) scales x by theta = omega^2/(omega^2 + a0),
    // the prefactor by sqrt(theta) and maps each node u -> u theta / (u + 1 -
    // u theta); omega < 0 (short range, erfc) visits every primitive quartet
    // twice, as the full operator and as the long-range one with weights
    // times -sqrt(theta), and skips it when theta x exceeds 40 or the
    // screening budget left.
    const double omega = prm.omega;
    const int reps = omega < 0.0 ? 2 : 1;
    bool run = false;
    // Pair records are loaded when used: loading the next quartet's records
    // one iteration ahead held 16 more doubles per lane and measured 7 %
    // slower on the sweep and 12 % slower on the FP32 Fock build.
    PrimPair bra, ket;
    // Fock mode, primitive screening: log(tau_prim / d) with d the quartet's
    // density factor (the same maximum the quartet screening uses)
    const bool pscreen = MODE == 1 && fk.lq != nullptr;
    float lthr = 0.f;
    if (MODE == 1 && pscreen && have) {
      const int nb = fk.nbas;
      const double *D = fk.Dsh;
      const int I = job.ish, J = job.jsh, K = job.ksh, L = job.lsh;
      const double dd = fmax(fmax(2.0 * D[I * nb + J], 2.0 * D[K * nb + L]),
                             fmax(fmax(D[I * nb + K], D[I * nb + L]), fmax(D[J * nb + K], D[J * nb + L])));
      lthr = dd > 0.0 ? (float)log(fk.tau_prim / dd) : INFINITY;
    }
    for (int it = 0; it < npmax * reps; ++it) {
      const bool lr_part = reps == 2 && (it & 1);
      const int p = reps == 2 ? (it >> 1) : it;
      if (!lr_part) run = p < np;
      if (run && !lr_part) {
        ket = prm.pp[job.pkl_off + kl];
        bra = prm.pp[job.pij_off + ij];
        const float lq2 = pscreen ? fk.lq[job.pij_off + ij] + fk.lq[job.pkl_off + kl] : 0.f;
        if constexpr (MODE == 0) {
          if (++ij == nbk) {
            ij = 0;
            ++kl;
            if (p + 1 < np) {
              const double kc = prm.pp[job.pkl_off + kl].cce;
              while (nbk > 0 && !(prm.pp[job.pij_off + nbk - 1].cce <= cut - kc)) --nbk;
            }
          }
        } else {
          // screening (reference src/cint2e.rs:367-393), then the primitive
          // Schwarz x density test
          run = !(ket.cce > cut) && !(bra.cce > cut - ket.cce);
          if (pscreen) run = run && lq2 >= lthr;
          if (++ij == job.nij) { ij = 0; ++kl; }
          nprim += run && rho == 0;
        }
      }
      // Roots, weights, prefactors and the per-unit coefficients are FP64 in
      // both variants and rounded once to R at the recurrence.
      double aij = 1.0, akl = 1.0, inv = 1.0, fac1 = 0.0, x = 0.0;
      double pq[3] = {0, 0, 0};
      if (run) {
        aij = bra.a; akl = ket.a;
        inv = 1.0 / (aij + akl);
        fac1 = sqrt(inv) * bra.facia * ket.facia;
        pq[0] = bra.px - ket.px; pq[1] = bra.py - ket.py; pq[2] = bra.pz - ket.pz;
        x = aij * akl * inv * (pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2]);
        double theta = 0.0;
        if (omega != 0.0) {
          theta = omega * omega / (omega * omega + aij * akl * inv);
          if (omega < 0.0 && !lr_part && theta * x > fmin(40.0, cut - bra.cce - ket.cce))
            run = false;                        // both parts of this primitive quartet
        }
        const bool attenuate = omega > 0.0 || lr_part;
        if (attenuate) {
          x *= theta;
          fac1 *= omega > 0.0 ? sqrt(theta) : -sqrt(theta);
        }
        if (run) {
          for (int f = rho; f < 2 * C::NR; f += C::LANES) {
            double v = rys_function<C::NR>(tab, x, f);
            if (attenuate && f < C::NR) v = v * theta / (v + 1.0 - v * theta);
            RW[f] = v;
            if (f < C::NR) RW[2 * C::NR + f] = 1.0 / (1.0 + v);   // t^2 complement 1/(1+u)
          }
        }
      }
      __syncwarp();
      if (run) {
        // rounds of (root, axis) units per lane, unrolled so that a lane's
        // independent units can interleave
        constexpr int UR = (3 * C::NR + C::LANES - 1) / C::LANES;
#pragma unroll
        for (int k = 0; k < UR; ++k) {
          const int u = rho + k * C::LANES;
          if (u >= 3 * C::NR) break;
          const int r = u / 3, ax = u - 3 * r;
          const double pa = pick3(bra.px - rA[0], bra.py - rA[1], bra.pz - rA[2], ax);
          const double qc = pick3(ket.px - rC[0], ket.py - rC[1], ket.pz - rC[2], ax);
          const double pqa = pick3(pq[0], pq[1], pq[2], ax);
          const double ab = pick3(rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2], ax);
          const double cd = pick3(rC[0] - rD[0], rC[1] - rD[1], rC[2] - rD[2], ax);
          // with d = 1/(1+u): B00 = u d / (2 (aij+akl)), B10 = B00 + d / (2 aij),
          // B01 = B00 + d / (2 akl) (u2 (aij+akl) + aij akl = aij akl (1+u))
          const double d = RW[2 * C::NR + r];
          const double tmp5 = 0.5 * inv * RW[r] * d;
          const double b10 = tmp5 + 0.5 * bra.ia * d;
          const double b01 = tmp5 + 0.5 * ket.ia * d;
          const double cn = pa - 2.0 * tmp5 * akl * pqa;
          const double cm = qc + 2.0 * tmp5 * aij * pqa;
          const double v00 = ax == 2 ? RW[C::NR + r] * fac1 : 1.0;
          vrr_hrr_unit<C, R>(G + (r * 3 + ax) * C::GST, Tsc + u * C::TST, (R)v00, (R)cn, (R)cm,
                             (R)b10, (R)b01, (R)tmp5, (R)ab, (R)cd);
        }
      }
      __syncwarp();
      if (run) {
#pragma unroll
        for (int r = 0; r < C::NR; ++r) {
          const R *gx = G + (r * 3 + 0) * C::GST, *gy = G + (r * 3 + 1) * C::GST;
          const R *gz = G + (r * 3 + 2) * C::GST;
          if (rho < C::NROWS) {
            R vx[C::CW], vy[C::CW], vz[C::CW];
#pragma unroll
            for (int m = 0; m < C::CW; ++m) {
              vx[m] = gx[roff[0] + m]; vy[m] = gy[roff[1] + m]; vz[m] = gz[roff[2] + m];
            }
            gout_cols<C, R, 0>(acc, vx, vy, vz);
          }
          if constexpr (C::NEX > 0) {
#pragma unroll
            for (int k = 0; k < C::NEX; ++k)
              if (xrow[k] >= 0) xacc[k] = fma(gx[xoff[k][0]] * gy[xoff[k][1]], gz[xoff[k][2]], xacc[k]);
          }
        }
      }
      __syncwarp();
    }

    // ---------------------------------------------------------- epilogue
    R *Bk = reinterpret_cast<R *>(sb);           // cartesian block, canonical
    if (have) {
      if (rho < C::NROWS) {
#pragma unroll
        for (int c = 0; c < C::NCOLS; ++c)
          Bk[C::ROWKET ? c + C::NBRA * rho : rho + C::NBRA * c] = acc[c];
      }
      if constexpr (C::NEX > 0) {
#pragma unroll
        for (int k = 0; k < C::NEX; ++k) {
          if (xrow[k] < 0) continue;
          const int e = rho + C::LANES * k, col = e % C::NCOLS;
          Bk[C::ROWKET ? col + C::NBRA * xrow[k] : xrow[k] + C::NBRA * col] = xacc[k];
        }
      }
    }
    __syncwarp();
    // Every warp barrier below is reached by all 32 lanes: lanes without a
    // job (the tail of the last task) skip only the work, never a barrier.
    R *T2 = Bk + C::NBRA * C::NKET;
    if (MODE == 0 && have) {
      // ket transform: T2[bra cart][ket out] (identity when cartesian)
      for (int t = rho; t < C::NBRA * NKO; t += C::LANES) {
        const int kap = t / C::NBRA, bc = t - kap * C::NBRA;
        const int ko = kap % NKo, lo = kap / NKo;
        R v = 0;
        if (!sph) {
          v = Bk[bc + C::NBRA * (ko + C::NK * lo)];
        } else {
          for (int kc = 0; kc < C::NK; ++kc) {
            const double ck = LK < 2 ? (kc == ko ? 1.0 : 0.0) : c2s_s[(LK * 5 + ko) * 6 + kc];
            if (ck == 0.0) continue;
            for (int lc = 0; lc < C::NL; ++lc) {
              const double cl = LL < 2 ? (lc == lo ? 1.0 : 0.0) : c2s_s[(LL * 5 + lo) * 6 + lc];
              if (cl == 0.0) continue;
              v = fma((R)(ck * cl), Bk[bc + C::NBRA * (kc + C::NK * lc)], v);
            }
          }
        }
        T2[t] = v;
      }
    }
    if (MODE == 0) __syncwarp();
    if (MODE == 0 && have) {
      // bra transform and store (i fastest -> coalesced for canonical order)
      for (int t = rho; t < NBO * NKO; t += C::LANES) {
        const int kap = t / NBO, b = t - kap * NBO;
        const int io = b % NIo, jo = b / NIo;
        const int ko = kap % NKo, lo = kap / NKo;
        R v = 0;
        if (!sph) {
          v = T2[io + C::NI * jo + C::NBRA * kap];
        } else {
          for (int ic = 0; ic < C::NI; ++ic) {
            const double ci = LI < 2 ? (ic == io ? 1.0 : 0.0) : c2s_s[(LI * 5 + io) * 6 + ic];
            if (ci == 0.0) continue;
            for (int jc = 0; jc < C::NJ; ++jc) {
              const double cj = LJ < 2 ? (jc == jo ? 1.0 : 0.0) : c2s_s[(LJ * 5 + jo) * 6 + jc];
              if (cj == 0.0) continue;
              v = fma((R)(ci * cj), T2[ic + C::NI * jc + C::NBRA * kap], v);
            }
          }
        }
        prm.out[job.out_off + (long long)io * job.s_i + (long long)jo * job.s_j +
                (long long)ko * job.s_k + (long long)lo * job.s_l] = (double)v;
      }
    }
    if constexpr (MODE == 1) {
      // staged density blocks start on an 8-byte boundary after the block
      R *Ps = reinterpret_cast<R *>(sb + RD_(C::NBRA * C::NKET * sizeof(R)));
      if (have) fock_stage<C::NI, C::NJ, C::NK, C::NL, R>(Ps, job, fk, rho, C::LANES);
      __syncwarp();
      if (have) fock_digest<C::NI, C::NJ, C::NK, C::NL, R>(Bk, Ps, job, wdeg, fk, rho, C::LANES);
    }
    __syncwarp();
  }
  if (MODE == 1 && fk.prim_count) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nprim += __shfl_xor_sync(0xffffffffu, nprim, o);
    if (lane == 0 && nprim) atomicAdd(fk.prim_count, nprim);
  }
}

// ---------------------------------------------------------------- lane per primitive quartet
// Fock-mode kernel for the small classes and shell quartets with at least
// LP_MIN_PRIM primitive quartets: one warp takes one shell quartet and each
// lane runs whole primitive quartets -- nodes, the recurrences of every
// (root, axis) and the block products -- in its own registers, with no
// shared memory or warp barrier per primitive quartet.  The block is summed
// across the lanes with shuffles once per shell quartet and digested like
// the slot kernels do.  Blocks of more than LP_CHUNK elements are made in
// passes of at most LP_CHUNK accumulators each, every pass recomputing the
// recurrences (registers bound the accumulators).  The classes: at most 27
// cartesian elements ((ss|ss) .. (dp|ss), one pass), (ds|pp) and (ds|ds) in
// 2 passes and, FP64 only, (pp|pp) in 3: the classes and precisions where
// the C3 cluster's build measured faster than on the slot kernel ((pp|pp)
// FP32 and (dp|ps) in 2 passes measured 22 % and 4-31 % slower).
constexpr int LP_CHUNK = 27;
constexpr int LP_MIN_PRIM = 32;

template <int LI, int LJ, int LK, int LL, typename R>
constexpr int lp_passes() {
  constexpr int ne = ncart(LI) * ncart(LJ) * ncart(LK) * ncart(LL);
  if (ne <= LP_CHUNK) return 1;
  if (LI == 2 && LJ == 0 && ((LK == 1 && LL == 1) || (LK == 2 && LL == 0))) return 2;
  if (LI == 1 && LJ == 1 && LK == 1 && LL == 1 && sizeof(R) == 8) return 3;
  return 0;
}

// offset of element (i, j, k, l) in one axis' G block (vrr_hrr_unit layout)
template <class C>
constexpr int lp_off(int i, int j, int k, int l, int ax) {
  return C::ROWKET ? C::ket_off(k, l, ax) * C::BSZ + C::bra_off(i, j, ax)
                   : C::bra_off(i, j, ax) * C::KSZ + C::ket_off(k, l, ax);
}

// acc[E - E0] += x y z for the elements E0 <= E < E1 of the canonical block,
// E = i + NI (j + NJ (k + NK l))
template <class C, typename R, int E0, int E1, int E, int NA>
__device__ __forceinline__ void lp_gout(R (&acc)[NA], const R (&gx)[C::GSZ], const R (&gy)[C::GSZ],
                                        const R (&gz)[C::GSZ]) {
  if constexpr (E < E1) {
    constexpr int i = E % C::NI, j = (E / C::NI) % C::NJ, k = (E / C::NBRA) % C::NK;
    constexpr int l = E / (C::NBRA * C::NK);
    constexpr int X = lp_off<C>(i, j, k, l, 0), Y = lp_off<C>(i, j, k, l, 1);
    constexpr int Z = lp_off<C>(i, j, k, l, 2);
    acc[E - E0] = fma(gx[X] * gy[Y], gz[Z], acc[E - E0]);
    lp_gout<C, R, E0, E1, E + 1, NA>(acc, gx, gy, gz);
  }
}

template <int LI, int LJ, int LK, int LL, typename R>
struct LpLayout {
  using C = EriClass<LI, LJ, LK, LL, true>;
  using S = FockStage<C::NI, C::NJ, C::NK, C::NL>;
  static constexpr int NE = C::NBRA * C::NKET;
  static constexpr int NPASS = lp_passes<LI, LJ, LK, LL, R>();
  static constexpr int CH = (NE + NPASS - 1) / NPASS;   // accumulators per pass
  static constexpr int TAB = RYS_TAB_OFFSET[C::NR + 1] - RYS_TAB_OFFSET[C::NR];
  static constexpr int WAREA = RD_(NE * sizeof(R)) + RD_(S::SIZE * sizeof(R)) + 1;   // doubles
  static constexpr size_t SMEM = sizeof(double) * (size_t)(TAB + ERI_WARPS * WAREA);
};

// Per-quartet constants of the lane kernel.
struct LpQuartet {
  QuartetJob job;
  double rA[3], rB[3], rC[3], rD[3];
  float lthr;
  int np;
};

// One pass: elements [PASS * CH, min(NE, (PASS + 1) * CH)) of the block,
// summed over this lane's primitive quartets, then over the warp, into Bk.
template <class C, class Lay, typename R, int PASS>
__device__ __forceinline__ void lp_pass(const EriParams &prm, const FockParams &fk, const double *tab,
                                        const LpQuartet &q, R *Bk, int lane, unsigned long long &nprim) {
  constexpr int NE = Lay::NE, NR = C::NR, CH = Lay::CH;
  constexpr int E0 = PASS * CH, E1 = (PASS + 1) * CH < NE ? (PASS + 1) * CH : NE;
  const double cut = prm.expcutoff, omega = prm.omega;
  const int reps = omega < 0.0 ? 2 : 1;
  const QuartetJob &job = q.job;
  R acc[CH];
#pragma unroll
  for (int e = 0; e < CH; ++e) acc[e] = 0;
  for (int p = lane; p < q.np; p += 32) {
    const int ij = p % job.nij, kl = p / job.nij;
    const PrimPair ket = prm.pp[job.pkl_off + kl];
    const PrimPair bra = prm.pp[job.pij_off + ij];
    // screening (reference src/cint2e.rs:367-393), then the primitive
    // Schwarz x density test
    if (ket.cce > cut || bra.cce > cut - ket.cce) continue;
    if (fk.lq && fk.lq[job.pij_off + ij] + fk.lq[job.pkl_off + kl] < q.lthr) continue;
    const double aij = bra.a, akl = ket.a, inv = 1.0 / (aij + akl);
    const double fac0 = sqrt(inv) * bra.facia * ket.facia;
    const double pq[3] = {bra.px - ket.px, bra.py - ket.py, bra.pz - ket.pz};
    const double x0 = aij * akl * inv * (pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2]);
    const double theta = omega != 0.0 ? omega * omega / (omega * omega + aij * akl * inv) : 0.0;
    if (omega < 0.0 && theta * x0 > fmin(40.0, cut - bra.cce - ket.cce)) continue;
    if (PASS == 0) ++nprim;
    const double pa[3] = {bra.px - q.rA[0], bra.py - q.rA[1], bra.pz - q.rA[2]};
    const double qc[3] = {ket.px - q.rC[0], ket.py - q.rC[1], ket.pz - q.rC[2]};
    for (int part = 0; part < reps; ++part) {
      // range separation as in k_eri (omega = env[8])
      const bool attenuate = omega > 0.0 || part == 1;
      const double x = attenuate ? x0 * theta : x0;
      const double fac1 = attenuate ? fac0 * (omega > 0.0 ? sqrt(theta) : -sqrt(theta)) : fac0;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double u = rys_function<NR>(tab, x, r);
        const double w = rys_function<NR>(tab, x, NR + r);
        if (attenuate) u = u * theta / (u + 1.0 - u * theta);
        const double d = 1.0 / (1.0 + u);
        const double tmp5 = 0.5 * inv * u * d;
        const double b10 = tmp5 + 0.5 * bra.ia * d;
        const double b01 = tmp5 + 0.5 * ket.ia * d;
        R g[3][C::GSZ];
        R tsc[C::TSZ > 0 ? C::TSZ : 1];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          const double cn = pa[ax] - 2.0 * tmp5 * akl * pq[ax];
          const double cm = qc[ax] + 2.0 * tmp5 * aij * pq[ax];
          const double v00 = ax == 2 ? w * fac1 : 1.0;
          vrr_hrr_unit<C, R>(g[ax], tsc, (R)v00, (R)cn, (R)cm, (R)b10, (R)b01, (R)tmp5,
                             (R)(q.rA[ax] - q.rB[ax]), (R)(q.rC[ax] - q.rD[ax]));
        }
        lp_gout<C, R, E0, E1, E0, CH>(acc, g[0], g[1], g[2]);
      }
    }
  }
  // sum over the lanes; lane e % 32 stores element E0 + e
#pragma unroll
  for (int e = 0; e < E1 - E0; ++e) {
    R v = acc[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((e & 31) == lane) Bk[E0 + e] = v;
  }
  if constexpr (PASS + 1 < Lay::NPASS) lp_pass<C, Lay, R, PASS + 1>(prm, fk, tab, q, Bk, lane, nprim);
}

template <int LI, int LJ, int LK, int LL, typename R>
__global__ void __launch_bounds__(ERI_THREADS)
k_fock_lp(EriParams prm, FockParams fk, const double *__restrict__ rys_tab_n, int *counter) {
  using Lay = LpLayout<LI, LJ, LK, LL, R>;
  using C = typename Lay::C;
  constexpr int NE = Lay::NE;
  static_assert(Lay::NPASS > 0, "not a lane-kernel class");
  extern __shared__ double smem[];
  double *tab = smem;
  for (int i = threadIdx.x; i < Lay::TAB; i += blockDim.x) tab[i] = rys_tab_n[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *wa = smem + Lay::TAB + warp * Lay::WAREA;
  R *Bk = reinterpret_cast<R *>(wa);
  R *Ps = reinterpret_cast<R *>(wa + RD_(NE * sizeof(R)));
  unsigned long long nprim = 0;
  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(counter, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= prm.njobs) break;
    const int2 jb = fk.jobs[prm.order[task]];
    const PairInfo pb = fk.pairs[jb.x], pk = fk.pairs[jb.y];
    LpQuartet q;
    QuartetJob &job = q.job;
    job.ish = pb.ish; job.jsh = pb.jsh; job.pij_off = pb.pp_off; job.nij = pb.npp;
    job.ksh = pk.ish; job.lsh = pk.jsh; job.pkl_off = pk.pp_off; job.nkl = pk.npp;
    job.out_off = 0; job.s_i = job.s_j = job.s_k = job.s_l = 0;
    q.np = job.nij * job.nkl;
    double wdeg = 1.0;
    if (pb.ish == pb.jsh) wdeg *= 0.5;
    if (pk.ish == pk.jsh) wdeg *= 0.5;
    if (jb.x == jb.y) wdeg *= 0.5;
    {
      const int a = C::IB ? job.ish : job.jsh, b = C::IB ? job.jsh : job.ish;
      const int c = C::KB ? job.ksh : job.lsh, d = C::KB ? job.lsh : job.ksh;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        q.rA[x] = prm.centers[3 * a + x]; q.rB[x] = prm.centers[3 * b + x];
        q.rC[x] = prm.centers[3 * c + x]; q.rD[x] = prm.centers[3 * d + x];
      }
    }
    q.lthr = 0.f;
    if (fk.lq) {
      const int nb = fk.nbas;
      const double *D = fk.Dsh;
      const int I = job.ish, J = job.jsh, K = job.ksh, L = job.lsh;
      const double dd = fmax(fmax(2.0 * D[I * nb + J], 2.0 * D[K * nb + L]),
                             fmax(fmax(D[I * nb + K], D[I * nb + L]), fmax(D[J * nb + K], D[J * nb + L])));
      q.lthr = dd > 0.0 ? (float)log(fk.tau_prim / dd) : INFINITY;
    }
    lp_pass<C, Lay, R, 0>(prm, fk, tab, q, Bk, lane, nprim);
    fock_stage<C::NI, C::NJ, C::NK, C::NL, R>(Ps, job, fk, lane, 32);
    __syncwarp();
    fock_digest<C::NI, C::NJ, C::NK, C::NL, R>(Bk, Ps, job, wdeg, fk, lane, 32);
    __syncwarp();
  }
  if (fk.prim_count) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nprim += __shfl_xor_sync(0xffffffffu, nprim, o);
    if (lane == 0 && nprim) atomicAdd(fk.prim_count, nprim);
  }
}

}  // namespace lrb
