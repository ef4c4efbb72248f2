// Rys ERI kernel for the classes with an f shell (l = 3): one shell quartet
// per CTA, class sizes at run time.
//
// The templated kernels (eri_kernel.cuh) keep a row of the cartesian block in
// each lane's registers, which stops fitting once a shell carries 10
// cartesian functions.  Here the whole CTA works on one quartet and keeps the
// block in shared memory:
//   * per primitive quartet: threads 0..2n_r-1 evaluate the Rys nodes and
//     weights (the same piecewise tables), threads 0..3n_r-1 run one
//     (root, axis) unit each -- the 2D VRR on the base centres and both
//     horizontal shifts (reference src/g2e.rs:316-909, the same recurrences as
//     vrr_hrr_unit) -- and then every thread accumulates its share of the
//     block, I(e) += sum_r Gx Gy Gz (src/cint2e.rs:2456-2895), through a
//     per-class table of packed (x, y, z) offsets;
//   * the epilogue transforms to spherical harmonics and writes the libcint
//     block (output mode) or digests the cartesian block into J/K (Fock
//     mode), as the templated kernels do.
// Screening is the reference's per primitive quartet (src/cint2e.rs:367-393).
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "eri_classes.cuh"

namespace lrb {

namespace {

constexpr int GEN_LMAX = 3;
constexpr int GEN_NAB = 2 * GEN_LMAX;   // largest la + lb

__device__ __forceinline__ double rys_function_rt(const double *tab, int nr, double x, int f) {
  switch (nr) {
    case 1: return rys_function<1>(tab, x, f);
    case 2: return rys_function<2>(tab, x, f);
    case 3: return rys_function<3>(tab, x, f);
    case 4: return rys_function<4>(tab, x, f);
    case 5: return rys_function<5>(tab, x, f);
    case 6: return rys_function<6>(tab, x, f);
    default: return rys_function<7>(tab, x, f);
  }
}

__device__ __forceinline__ void comp_of(int l, int n, int &x, int &y, int &z) {
  int t = 0;
  while ((t + 1) * (t + 2) / 2 <= n) ++t;
  z = n - t * (t + 1) / 2;
  y = t - z;
  x = l - t;
}

__device__ __forceinline__ double c2s_coef(int l, int m, int c) {
  return l < 2 ? (m == c ? 1.0 : 0.0) : c_c2s[(l * C2S_M + m) * C2S_C + c];
}

// One (root, axis) unit: G[a][b][c][d] ((a*(lb+1)+b)*(lc+1)+c)*(ld+1)+d.
__device__ void gen_unit(const GenClass &g, double *G, double v00, double cn, double cm, double b10,
                         double b01, double b00, double ab, double cd) {
  double v[GEN_NAB + 1][GEN_NAB + 1];
  const int nab = g.la + g.lb, ncd = g.lc + g.ld;
  v[0][0] = v00;
  for (int m = 1; m <= ncd; ++m) {
    double t = cm * v[0][m - 1];
    if (m > 1) t = fma((m - 1) * b01, v[0][m - 2], t);
    v[0][m] = t;
  }
  for (int n = 1; n <= nab; ++n)
    for (int m = 0; m <= ncd; ++m) {
      double t = cn * v[n - 1][m];
      if (n > 1) t = fma((n - 1) * b10, v[n - 2][m], t);
      if (m > 0) t = fma(m * b00, v[n - 1][m - 1], t);
      v[n][m] = t;
    }
  // bra shift, in place per m: column b of v[.][m] holds h[a][b]
  double T[GEN_LMAX + 1][GEN_LMAX + 1][GEN_NAB + 1];
  for (int m = 0; m <= ncd; ++m) {
    double h[GEN_NAB + 1];
    for (int n = 0; n <= nab; ++n) h[n] = v[n][m];
    for (int a = 0; a <= g.la; ++a) T[a][0][m] = h[a];
    for (int b = 1; b <= g.lb; ++b) {
      for (int a = 0; a <= nab - b; ++a) h[a] = fma(ab, h[a], h[a + 1]);
      for (int a = 0; a <= g.la; ++a) T[a][b][m] = h[a];
    }
  }
  for (int a = 0; a <= g.la; ++a)
    for (int b = 0; b <= g.lb; ++b) {
      double k[GEN_NAB + 1];
      for (int m = 0; m <= ncd; ++m) k[m] = T[a][b][m];
      double *o = G + (a * (g.lb + 1) + b) * (g.lc + 1) * (g.ld + 1);
      for (int c = 0; c <= g.lc; ++c) o[c * (g.ld + 1)] = k[c];
      for (int d = 1; d <= g.ld; ++d) {
        for (int c = 0; c <= ncd - d; ++c) k[c] = fma(cd, k[c], k[c + 1]);
        for (int c = 0; c <= g.lc; ++c) o[c * (g.ld + 1) + d] = k[c];
      }
    }
}

// J/K digestion of a cartesian block (the templated fock_digest with run-time
// sizes): B[a + ni*(b + nj*(c + nk*d))], degeneracy weight w.
__device__ void gen_digest(const double *B, const QuartetJob &q, double w, const FockParams &fk,
                           int ni, int nj, int nk, int nl, int tid, int nt) {
  const int n = fk.n;
  const int oi = fk.aooff[q.ish], oj = fk.aooff[q.jsh], ok = fk.aooff[q.ksh], ol = fk.aooff[q.lsh];
  const double *P = fk.P;
  auto blk = [&](int a, int b, int c, int d) { return B[a + ni * (b + nj * (c + nk * d))]; };
  auto p = [&](int r, int c) { return P[(long long)r * n + c]; };
  for (int t = tid; t < ni * nj; t += nt) {
    const int a = t % ni, b = t / ni;
    double s = 0;
    for (int d = 0; d < nl; ++d)
      for (int c = 0; c < nk; ++c) s = fma(blk(a, b, c, d), p(ok + c, ol + d), s);
    atomicAdd(&fk.J[(long long)(oi + a) * n + oj + b], 2.0 * w * s);
  }
  for (int t = tid; t < nk * nl; t += nt) {
    const int c = t % nk, d = t / nk;
    double s = 0;
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a) s = fma(blk(a, b, c, d), p(oi + a, oj + b), s);
    atomicAdd(&fk.J[(long long)(ok + c) * n + ol + d], 2.0 * w * s);
  }
  for (int t = tid; t < ni * nk; t += nt) {
    const int a = t % ni, c = t / ni;
    double s = 0;
    for (int d = 0; d < nl; ++d)
      for (int b = 0; b < nj; ++b) s = fma(blk(a, b, c, d), p(oj + b, ol + d), s);
    atomicAdd(&fk.K[(long long)(oi + a) * n + ok + c], w * s);
  }
  for (int t = tid; t < nj * nk; t += nt) {
    const int b = t % nj, c = t / nj;
    double s = 0;
    for (int d = 0; d < nl; ++d)
      for (int a = 0; a < ni; ++a) s = fma(blk(a, b, c, d), p(oi + a, ol + d), s);
    atomicAdd(&fk.K[(long long)(oj + b) * n + ok + c], w * s);
  }
  for (int t = tid; t < ni * nl; t += nt) {
    const int a = t % ni, d = t / ni;
    double s = 0;
    for (int c = 0; c < nk; ++c)
      for (int b = 0; b < nj; ++b) s = fma(blk(a, b, c, d), p(oj + b, ok + c), s);
    atomicAdd(&fk.K[(long long)(oi + a) * n + ol + d], w * s);
  }
  for (int t = tid; t < nj * nl; t += nt) {
    const int b = t % nj, d = t / nj;
    double s = 0;
    for (int c = 0; c < nk; ++c)
      for (int a = 0; a < ni; ++a) s = fma(blk(a, b, c, d), p(oi + a, ok + c), s);
    atomicAdd(&fk.K[(long long)(oj + b) * n + ol + d], w * s);
  }
}

}  // namespace

// Shared memory (doubles): rw[3 nr] | G[3 nr gsz] | acc[nbra nket] |
// tmp[nbra nsph(lk) nsph(ll)] (output mode) | packed offsets (nbra nket ints).
// (ff|ff) in output mode: 162 KB of doubles + 40 KB of offsets.
int gen_tmp_doubles(const GenClass &g, int mode) {
  return mode == 0 ? g.ni * g.nj * nsph(g.lk) * nsph(g.ll) : 0;
}
size_t gen_smem_bytes(const GenClass &g, int mode) {
  const size_t ne = (size_t)g.ni * g.nj * g.nk * g.nl;
  const size_t d = 3 * g.nr + 3 * (size_t)g.nr * g.gsz + ne + gen_tmp_doubles(g, mode);
  return d * sizeof(double) + ne * sizeof(int);
}

template <int MODE>
__global__ void __launch_bounds__(GEN_THREADS)
k_eri_gen(EriParams prm, FockParams fk, GenClass g, const double *__restrict__ rys_tab_n,
          int *counter) {
  extern __shared__ double smem[];
  const int nr = g.nr, gsz = g.gsz;
  const int ne = g.ni * g.nj * g.nk * g.nl, nbra = g.ni * g.nj;
  double *RW = smem;                       // [3 nr]
  double *G = RW + 3 * nr;                 // [nr][3][gsz]
  double *acc = G + 3 * nr * gsz;          // [ne]
  double *tmp = acc + ne;                  // output mode, spherical: ket-transformed block
  int *eoff = reinterpret_cast<int *>(tmp + (MODE == 0 ? g.ni * g.nj * nsph(g.lk) * nsph(g.ll) : 0));
  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ int s_task;

  // packed per-axis offsets of every element of the canonical block
  for (int e = tid; e < ne; e += nt) {
    const int i = e % g.ni, j = (e / g.ni) % g.nj, k = (e / nbra) % g.nk, l = e / (nbra * g.nk);
    int pi[3], pj[3], pk[3], pl[3];
    comp_of(g.li, i, pi[0], pi[1], pi[2]);
    comp_of(g.lj, j, pj[0], pj[1], pj[2]);
    comp_of(g.lk, k, pk[0], pk[1], pk[2]);
    comp_of(g.ll, l, pl[0], pl[1], pl[2]);
    int packed = 0;
    for (int ax = 0; ax < 3; ++ax) {
      const int a = g.ib ? pi[ax] : pj[ax], b = g.ib ? pj[ax] : pi[ax];
      const int c = g.kb ? pk[ax] : pl[ax], d = g.kb ? pl[ax] : pk[ax];
      packed |= (((a * (g.lb + 1) + b) * (g.lc + 1) + c) * (g.ld + 1) + d) << (10 * ax);
    }
    eoff[e] = packed;
  }
  const bool sph = MODE == 0 && prm.sph != 0;
  const int nio = sph ? nsph(g.li) : g.ni, njo = sph ? nsph(g.lj) : g.nj;
  const int nko = sph ? nsph(g.lk) : g.nk, nlo = sph ? nsph(g.ll) : g.nl;
  unsigned long long nprim = 0;

  for (;;) {
    __syncthreads();
    if (tid == 0) s_task = atomicAdd(counter, 1);
    __syncthreads();
    const int task = s_task;
    if (task >= prm.njobs) break;
    QuartetJob job;
    double wdeg = 1.0;
    if (MODE == 0) {
      job = prm.jobs[prm.order[task]];
    } else {
      const int2 jb = fk.jobs[prm.order[task]];
      const PairInfo pb = fk.pairs[jb.x], pk = fk.pairs[jb.y];
      job.ish = pb.ish; job.jsh = pb.jsh; job.pij_off = pb.pp_off; job.nij = pb.npp;
      job.ksh = pk.ish; job.lsh = pk.jsh; job.pkl_off = pk.pp_off; job.nkl = pk.npp;
      job.out_off = 0; job.s_i = job.s_j = job.s_k = job.s_l = 0;
      if (pb.ish == pb.jsh) wdeg *= 0.5;
      if (pk.ish == pk.jsh) wdeg *= 0.5;
      if (jb.x == jb.y) wdeg *= 0.5;
    }
    const int a = g.ib ? job.ish : job.jsh, b = g.ib ? job.jsh : job.ish;
    const int c = g.kb ? job.ksh : job.lsh, d = g.kb ? job.lsh : job.ksh;
    double rA[3], rB[3], rC[3], rD[3];
    for (int x = 0; x < 3; ++x) {
      rA[x] = prm.centers[3 * a + x]; rB[x] = prm.centers[3 * b + x];
      rC[x] = prm.centers[3 * c + x]; rD[x] = prm.centers[3 * d + x];
    }
    for (int e = tid; e < ne; e += nt) acc[e] = 0.0;
    const double cut = prm.expcutoff;
    // Fock mode, primitive screening (as the templated kernels)
    float lthr = -INFINITY;
    if (MODE == 1 && fk.lq) {
      const int nb = fk.nbas;
      const double *D = fk.Dsh;
      const int I = job.ish, J = job.jsh, K = job.ksh, L = job.lsh;
      const double dd = fmax(fmax(2.0 * D[I * nb + J], 2.0 * D[K * nb + L]),
                             fmax(fmax(D[I * nb + K], D[I * nb + L]), fmax(D[J * nb + K], D[J * nb + L])));
      lthr = dd > 0.0 ? (float)log(fk.tau_prim / dd) : INFINITY;
    }
    for (int kl = 0; kl < job.nkl; ++kl) {
      const PrimPair ket = prm.pp[job.pkl_off + kl];
      if (ket.cce > cut) continue;           // uniform over the CTA
      for (int ij = 0; ij < job.nij; ++ij) {
        const PrimPair bra = prm.pp[job.pij_off + ij];
        if (bra.cce > cut - ket.cce) continue;
        if (MODE == 1 && fk.lq && fk.lq[job.pij_off + ij] + fk.lq[job.pkl_off + kl] < lthr) continue;
        nprim += tid == 0;
        const double aij = bra.a, akl = ket.a, inv = 1.0 / (aij + akl);
        const double fac0 = sqrt(inv) * bra.facia * ket.facia;
        const double pq[3] = {bra.px - ket.px, bra.py - ket.py, bra.pz - ket.pz};
        const double x0 = aij * akl * inv * (pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2]);
        // range separation as in the templated kernels (omega = env[8])
        const double omega = prm.omega;
        const double theta = omega != 0.0 ? omega * omega / (omega * omega + aij * akl * inv) : 0.0;
        if (omega < 0.0 && theta * x0 > fmin(40.0, cut - bra.cce - ket.cce)) continue;
        for (int part = 0; part < (omega < 0.0 ? 2 : 1); ++part) {
        const bool attenuate = omega > 0.0 || part == 1;
        const double x = attenuate ? x0 * theta : x0;
        const double fac1 = attenuate ? fac0 * (omega > 0.0 ? sqrt(theta) : -sqrt(theta)) : fac0;
        __syncthreads();                      // previous primitive's G fully read
        if (tid < 2 * nr) {
          double v = rys_function_rt(rys_tab_n, nr, x, tid);
          if (attenuate && tid < nr) v = v * theta / (v + 1.0 - v * theta);
          RW[tid] = v;
          if (tid < nr) RW[2 * nr + tid] = 1.0 / (1.0 + v);
        }
        __syncthreads();
        if (tid < 3 * nr) {
          const int r = tid / 3, ax = tid - 3 * r;
          const double pp[3] = {bra.px, bra.py, bra.pz}, qq[3] = {ket.px, ket.py, ket.pz};
          const double dd = RW[2 * nr + r];
          const double tmp5 = 0.5 * inv * RW[r] * dd;
          const double b10 = tmp5 + 0.5 * bra.ia * dd;
          const double b01 = tmp5 + 0.5 * ket.ia * dd;
          const double cn = pp[ax] - rA[ax] - 2.0 * tmp5 * akl * pq[ax];
          const double cm = qq[ax] - rC[ax] + 2.0 * tmp5 * aij * pq[ax];
          const double v00 = ax == 2 ? RW[nr + r] * fac1 : 1.0;
          gen_unit(g, G + (r * 3 + ax) * gsz, v00, cn, cm, b10, b01, tmp5, rA[ax] - rB[ax],
                   rC[ax] - rD[ax]);
        }
        __syncthreads();
        for (int e = tid; e < ne; e += nt) {
          const int o = eoff[e];
          const int ox = o & 1023, oy = (o >> 10) & 1023, oz = o >> 20;
          double s = acc[e];
          for (int r = 0; r < nr; ++r) {
            const double *gr = G + r * 3 * gsz;
            s = fma(gr[ox] * gr[gsz + oy], gr[2 * gsz + oz], s);
          }
          acc[e] = s;
        }
        }   // parts
      }
    }
    __syncthreads();
    if (MODE == 0 && !sph) {
      for (int t = tid; t < ne; t += nt) {
        const int io = t % g.ni, jo = (t / g.ni) % g.nj, ko = (t / nbra) % g.nk, lo = t / (nbra * g.nk);
        prm.out[job.out_off + (long long)io * job.s_i + (long long)jo * job.s_j +
                (long long)ko * job.s_k + (long long)lo * job.s_l] = acc[t];
      }
    } else if (MODE == 0) {
      // ket transform tmp[bra cart + nbra * (ko + nko lo)], then bra and store
      for (int t = tid; t < nbra * nko * nlo; t += nt) {
        const int kap = t / nbra, bc = t - kap * nbra;
        const int ko = kap % nko, lo = kap / nko;
        double v = 0.0;
        for (int kc = 0; kc < g.nk; ++kc) {
          const double ck = c2s_coef(g.lk, ko, kc);
          if (ck == 0.0) continue;
          for (int lc = 0; lc < g.nl; ++lc) {
            const double cl = c2s_coef(g.ll, lo, lc);
            if (cl != 0.0) v = fma(ck * cl, acc[bc + nbra * (kc + g.nk * lc)], v);
          }
        }
        tmp[t] = v;
      }
      __syncthreads();
      const int nbo = nio * njo;
      for (int t = tid; t < nbo * nko * nlo; t += nt) {
        const int kap = t / nbo, bo = t - kap * nbo;
        const int io = bo % nio, jo = bo / nio;
        const int ko = kap % nko, lo = kap / nko;
        double v = 0.0;
        for (int ic = 0; ic < g.ni; ++ic) {
          const double ci = c2s_coef(g.li, io, ic);
          if (ci == 0.0) continue;
          for (int jc = 0; jc < g.nj; ++jc) {
            const double cj = c2s_coef(g.lj, jo, jc);
            if (cj != 0.0) v = fma(ci * cj, tmp[ic + g.ni * jc + nbra * kap], v);
          }
        }
        prm.out[job.out_off + (long long)io * job.s_i + (long long)jo * job.s_j +
                (long long)ko * job.s_k + (long long)lo * job.s_l] = v;
      }
    } else {
      gen_digest(acc, job, wdeg, fk, g.ni, g.nj, g.nk, g.nl, tid, nt);
    }
  }
  if (MODE == 1 && fk.prim_count && tid == 0 && nprim) atomicAdd(fk.prim_count, nprim);
}

GenClass gen_class(int li, int lj, int lk, int ll) {
  GenClass g;
  g.li = li; g.lj = lj; g.lk = lk; g.ll = ll;
  g.nr = (li + lj + lk + ll) / 2 + 1;
  g.ib = li > lj; g.kb = lk > ll;
  g.la = g.ib ? li : lj; g.lb = g.ib ? lj : li;
  g.lc = g.kb ? lk : ll; g.ld = g.kb ? ll : lk;
  g.ni = ncart(li); g.nj = ncart(lj); g.nk = ncart(lk); g.nl = ncart(ll);
  g.gsz = (g.la + 1) * (g.lb + 1) * (g.lc + 1) * (g.ld + 1);
  return g;
}

GenKernelFn gen_kernel(int mode) { return mode == 0 ? k_eri_gen<0> : k_eri_gen<1>; }

cudaError_t eri_register_gen(const double *c2s_host) {
  cudaError_t e = cudaMemcpyToSymbol(c_c2s, c2s_host, sizeof(c_c2s));
  // the largest class, (ff|ff), needs the most shared memory
  const GenClass big = gen_class(3, 3, 3, 3);
  for (int m = 0; m < 2 && e == cudaSuccess; ++m)
    e = cudaFuncSetAttribute(gen_kernel(m), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gen_smem_bytes(big, m));
  return e;
}

}  // namespace lrb
