// Batched ERI engine: quartet classification, primitive-pair preparation and
// per-class kernel launches.  All device work runs on the caller's stream.
#define RYS_TAB_QUAL __device__
#define RYS_CONST_QUAL __constant__
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "engine.h"
#include "eri_classes.cuh"

namespace lrb {

// ---------------------------------------------------------------- classes
// Canonical classes for l <= ERI_LMAX, id = P(P+1)/2 + Q with pair index
// P = li(li+1)/2 + lj of the bra (li >= lj) and Q of the ket, P >= Q.

// ---------------------------------------------------------------- prep
// One thread per quartet: canonical order, class key, block size, strides.
__global__ void k_classify(const int *__restrict__ shls, long long nq, const int *__restrict__ bas,
                           int nbas, int coord, QuartetJob *jobs, unsigned *keys, int *idx,
                           long long *blk, int *npair, int *err) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= nq) return;
  int s[4], l[4], k[4], n[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    s[a] = shls[4 * q + a];
    if (s[a] < 0 || s[a] >= nbas) {   // never dereference a bad shell index
      atomicExch(err, 2);
      s[a] = 0;
    }
    l[a] = bas[8 * s[a] + 1];
    k[a] = bas[8 * s[a] + 2];
    n[a] = coord == 0 ? ncart(l[a]) : nsph(l[a]);
    if (l[a] < 0 || l[a] > ERI_LMAX || k[a] < 1 || k[a] > ERI_KMAX || bas[8 * s[a] + 3] != 1)
      atomicExch(err, 1);
  }
  // original strides: out[i + ni*(j + nj*(k + nk*l))]
  const int st[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
  int p[4] = {0, 1, 2, 3};   // canonical position -> original position
  if (l[0] < l[1]) { p[0] = 1; p[1] = 0; }
  if (l[2] < l[3]) { p[2] = 3; p[3] = 2; }
  if (pair_index(l[p[0]], l[p[1]]) < pair_index(l[p[2]], l[p[3]])) {
    int t0 = p[0], t1 = p[1];
    p[0] = p[2]; p[1] = p[3]; p[2] = t0; p[3] = t1;
  }
  QuartetJob j;
  j.ish = s[p[0]]; j.jsh = s[p[1]]; j.ksh = s[p[2]]; j.lsh = s[p[3]];
  j.s_i = st[p[0]]; j.s_j = st[p[1]]; j.s_k = st[p[2]]; j.s_l = st[p[3]];
  j.nij = k[p[0]] * k[p[1]];
  j.nkl = k[p[2]] * k[p[3]];
  j.pij_off = 0; j.pkl_off = 0; j.out_off = 0;
  jobs[q] = j;
  const int cid = class_id(l[p[0]], l[p[1]], l[p[2]], l[p[3]]);
  const int kprod = j.nij * j.nkl;
  // class ascending, primitive count descending (big tasks first)
  keys[q] = ((unsigned)cid << 20) | (unsigned)(0xfffff - kprod);   // kprod <= 31^4 < 2^20
  idx[q] = (int)q;
  blk[q] = (long long)n[0] * n[1] * n[2] * n[3];
  npair[2 * q] = j.nij;
  npair[2 * q + 1] = j.nkl;
}

__global__ void k_offsets(QuartetJob *jobs, long long nq, const long long *out_off,
                          const int *pair_off) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= nq) return;
  jobs[q].out_off = out_off[q];
  jobs[q].pij_off = pair_off[2 * q];
  jobs[q].pkl_off = pair_off[2 * q + 1];
}

__device__ inline double common_fac_sp(int l) {
  return l == 0 ? 0.28209479177387814 : (l == 1 ? 0.48860251190291992 : 1.0);  // 1/sqrt(4pi), sqrt(3/(4pi))
}

// Primitive pair e (ip fastest) of shells (si, sj); ket pairs carry the
// class prefactor.  Screening key as CINTset_pairdata (reference
// src/optimizer.rs:732-808).
__device__ __forceinline__ PrimPair make_pair(int si, int sj, bool ket, int e,
                                              const int *__restrict__ atm,
                                              const int *__restrict__ bas,
                                              const double *__restrict__ env, int gc_screen) {
  const int *bi = bas + 8 * si, *bj = bas + 8 * sj;
  const int ki = bi[2], kj = bj[2];
  const int ip = e % ki, jp = e / ki;
  const double *ri = env + atm[6 * bi[0] + 1], *rj = env + atm[6 * bj[0] + 1];
  const double ai = env[bi[5] + ip], aj = env[bj[5] + jp];
  const double ci = env[bi[6] + ip], cj = env[bj[6] + jp];
  const double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
  const double rr = dx * dx + dy * dy + dz * dz;
  const double aij = ai + aj, inv = 1.0 / aij;
  const double eij = rr * ai * aj * inv;
  const int lij = bi[1] + bj[1];
  double log_rr = 1.7 - 1.5 * log(env[bi[5] + ki - 1] + env[bj[5] + kj - 1]);
  if (lij > 0) log_rr += lij * log(sqrt(rr) + 1.0);
  PrimPair o;
  o.a = aij;
  const double wj = aj * inv;
  o.px = ri[0] + wj * (rj[0] - ri[0]);
  o.py = ri[1] + wj * (rj[1] - ri[1]);
  o.pz = ri[2] + wj * (rj[2] - ri[2]);
  double fac = ci * cj * exp(-eij) * common_fac_sp(bi[1]) * common_fac_sp(bj[1]);
  // 2 pi^3 / sqrt(pi) = 2 pi^2.5 (reference src/g2e.rs:74-82), on the ket side
  if (ket) fac *= 34.986836655249725;
  o.fac = fac;
  o.ia = inv;
  o.facia = fac * inv;
  // sub-shells of a generally contracted shell screen with the largest
  // |coefficient| over its contractions (bas slot 7 when gc_screen)
  const double si_c = gc_screen && bi[7] > 0 ? env[bi[7] + ip] : ci;
  const double sj_c = gc_screen && bj[7] > 0 ? env[bj[7] + jp] : cj;
  o.cce = eij - log_rr - log(fabs(si_c)) - log(fabs(sj_c));
  return o;
}

// One warp sorts shell pair pr (pair 2q is the bra (i,j) of quartet q,
// 2q+1 the ket): builds its primitive pairs in natural order in `raw`, then
// writes each at its rank by ascending screening key (NaN last, ties by
// position), so the ERI kernel can visit only the passing prefix.
__device__ void pair_sort_warp(long long pr, int lane, const QuartetJob *__restrict__ jobs,
                               const int *__restrict__ pair_off, const int *__restrict__ atm,
                               const int *__restrict__ bas, const double *__restrict__ env,
                               PrimPair *__restrict__ pp, PrimPair *__restrict__ raw,
                               int gc_screen) {
  const QuartetJob j = jobs[pr >> 1];
  const bool ket = pr & 1;
  const int si = ket ? j.ksh : j.ish, sj = ket ? j.lsh : j.jsh;
  const int n = ket ? j.nkl : j.nij;
  const long long off = pair_off[pr];
  for (int e = lane; e < n; e += 32)
    raw[off + e] = make_pair(si, sj, ket, e, atm, bas, env, gc_screen);
  __syncwarp();
  for (int e = lane; e < n; e += 32) {
    const double c = cce_key(raw[off + e].cce);
    int rank = 0;
    for (int u = 0; u < n; ++u) {
      const double cu = cce_key(raw[off + u].cce);
      rank += (cu < c) || (cu == c && u < e);
    }
    pp[off + rank] = raw[off + e];
  }
}

// Shell-pair constants of one block's pairs, staged once per pair so every
// primitive of the pair needs only its four exponent/coefficient loads.
struct PairHead {
  double rix, riy, riz;   // centre of shell i
  double dx, dy, dz;      // R_j - R_i
  double rr, log_rr, cfac;
  int ea, ca, eb, cb;     // env offsets of exponents / coefficients of i and j
  int sa, sb;             // env offsets of the screening coefficients of i and j
  int ki, first;          // primitives of i; first primitive pair (block-relative)
};

constexpr int PB_PAIRS = 64;      // shell pairs per block
constexpr int PB_THREADS = 256;
constexpr int PB_CAP = 4096;      // primitive pairs per block ranked through shared memory

// Block of PB_PAIRS consecutive shell pairs: pass 1 writes every primitive
// pair's screening key (the same expression as make_pair) to shared memory
// with one thread per primitive pair, pass 2 rebuilds the pair and stores it
// at its rank within its shell pair (ascending key, NaN last, ties by
// position: the order pair_sort_warp produces).  Blocks whose primitive
// pairs exceed PB_CAP sort warp by warp instead.
__global__ void __launch_bounds__(PB_THREADS, 3)
k_pairs_block(const QuartetJob *__restrict__ jobs, long long nq, const int *__restrict__ npair,
              const int *__restrict__ pair_off, const int *__restrict__ atm,
              const int *__restrict__ bas, const double *__restrict__ env,
              PrimPair *__restrict__ pp, PrimPair *__restrict__ raw, int gc_screen) {
  __shared__ double skey[PB_CAP];
  __shared__ PairHead head[PB_PAIRS];
  __shared__ int soff[PB_PAIRS + 1];
  const long long p0 = (long long)blockIdx.x * PB_PAIRS;
  const int P = (int)min((long long)PB_PAIRS, 2 * nq - p0);
  const int t = threadIdx.x;
  if (t < P) {
    const long long pr = p0 + t;
    soff[t] = pair_off[pr];
    if (t == P - 1) soff[P] = pair_off[pr] + npair[pr];
    const QuartetJob j = jobs[pr >> 1];
    const bool ket = pr & 1;
    const int *bi = bas + 8 * (ket ? j.ksh : j.ish), *bj = bas + 8 * (ket ? j.lsh : j.jsh);
    const int ki = bi[2], kj = bj[2];
    const double *ri = env + atm[6 * bi[0] + 1], *rj = env + atm[6 * bj[0] + 1];
    PairHead h;
    h.rix = ri[0]; h.riy = ri[1]; h.riz = ri[2];
    h.dx = ri[0] - rj[0]; h.dy = ri[1] - rj[1]; h.dz = ri[2] - rj[2];
    h.rr = h.dx * h.dx + h.dy * h.dy + h.dz * h.dz;
    h.dx = rj[0] - ri[0]; h.dy = rj[1] - ri[1]; h.dz = rj[2] - ri[2];
    h.ea = bi[5]; h.ca = bi[6]; h.eb = bj[5]; h.cb = bj[6]; h.ki = ki;
    h.sa = gc_screen && bi[7] > 0 ? bi[7] : bi[6];
    h.sb = gc_screen && bj[7] > 0 ? bj[7] : bj[6];
    const int lij = bi[1] + bj[1];
    double log_rr = 1.7 - 1.5 * log(env[bi[5] + ki - 1] + env[bj[5] + kj - 1]);
    if (lij > 0) log_rr += lij * log(sqrt(h.rr) + 1.0);
    h.log_rr = log_rr;
    // 2 pi^3 / sqrt(pi) = 2 pi^2.5 (reference src/g2e.rs:74-82), on the ket side
    h.cfac = common_fac_sp(bi[1]) * common_fac_sp(bj[1]) * (ket ? 34.986836655249725 : 1.0);
    head[t] = h;
  }
  __syncthreads();
  const int base = soff[0], R = soff[P] - base;
  if (R > PB_CAP) {
    for (int w = t >> 5; w < P; w += PB_THREADS / 32)
      pair_sort_warp(p0 + w, t & 31, jobs, pair_off, atm, bas, env, pp, raw, gc_screen);
    return;
  }
  if (t < P) head[t].first = soff[t] - base;
  __syncthreads();
  // local shell pair of block-relative primitive pair e
  auto find = [&](int e) {
    int lo = 0, hi = P - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (soff[mid] - base <= e) lo = mid; else hi = mid - 1;
    }
    return lo;
  };
  for (int e = t; e < R; e += PB_THREADS) {
    const PairHead &h = head[find(e)];
    const int k = e - h.first, ip = k % h.ki, jp = k / h.ki;
    const double ai = env[h.ea + ip], aj = env[h.eb + jp];
    const double ci = env[h.sa + ip], cj = env[h.sb + jp];
    const double inv = 1.0 / (ai + aj);
    const double eij = h.rr * ai * aj * inv;
    skey[e] = eij - h.log_rr - log(fabs(ci)) - log(fabs(cj));
  }
  __syncthreads();
  for (int e = t; e < R; e += PB_THREADS) {
    const int p = find(e);
    const PairHead &h = head[p];
    const int k = e - h.first, ip = k % h.ki, jp = k / h.ki;
    const double ai = env[h.ea + ip], aj = env[h.eb + jp];
    const double ci = env[h.ca + ip], cj = env[h.cb + jp];
    const double aij = ai + aj, inv = 1.0 / aij;
    const double eij = h.rr * ai * aj * inv;
    const double wj = aj * inv;
    PrimPair o;
    o.a = aij;
    o.px = h.rix + wj * h.dx;
    o.py = h.riy + wj * h.dy;
    o.pz = h.riz + wj * h.dz;
    const double fac = ci * cj * exp(-eij) * h.cfac;
    o.fac = fac;
    o.ia = inv;
    o.facia = fac * inv;
    o.cce = skey[e];
    const double c = cce_key(o.cce);
    const int n = (p + 1 < P ? head[p + 1].first : R) - h.first;
    int rank = 0;
    for (int u = 0; u < n; ++u) {
      const double cu = cce_key(skey[h.first + u]);
      rank += (cu < c) || (cu == c && u < k);
    }
    pp[base + h.first + rank] = o;
  }
}

// Shell centres, with the bounds of every index a shell carries checked
// against natm / nenv so later kernels never read outside the inputs.
__global__ void k_centers(const int *__restrict__ atm, int natm, const int *__restrict__ bas,
                          int nbas, const double *__restrict__ env, long long nenv,
                          double *centers, int *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nbas) return;
  const int *b = bas + 8 * s;
  const int a = b[0], l = b[1], k = b[2], nctr = b[3];
  bool ok = a >= 0 && a < natm && l >= 0 && k >= 1 && nctr >= 1 && b[5] >= 0 && b[6] >= 0 &&
            (long long)b[5] + k <= nenv && (long long)b[6] + (long long)k * nctr <= nenv;
  const int pr = ok ? atm[6 * a + 1] : 0;
  ok = ok && pr >= 0 && (long long)pr + 3 <= nenv;
  if (!ok) {
    atomicExch(err, 2);
    centers[3 * s] = centers[3 * s + 1] = centers[3 * s + 2] = 0.0;
    return;
  }
  const double *r = env + pr;
  centers[3 * s] = r[0]; centers[3 * s + 1] = r[1]; centers[3 * s + 2] = r[2];
}

// First sorted position of every class (keys sorted ascending by class).
__global__ void k_class_starts(const unsigned *__restrict__ keys, long long nq, long long *starts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > NCLASS) return;
  long long lo = 0, hi = nq;
  const unsigned key = (unsigned)c << 20;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  starts[c] = lo;
}

// ---------------------------------------------------------------- dispatch
// Real solid harmonics as cartesian combinations, libcint order and
// normalisation: closed form of Helgaker, Jorgensen & Olsen, "Molecular
// Electronic-Structure Theory", eqs. 6.4.47-6.4.50, scaled by
// sqrt((2l+1)/(4 pi)); s and p are the identity (p kept as x, y, z), the
// reference's table is src/cart2sph.rs:26.
void fill_c2s(double *c) {
  auto fact = [](int n) { double r = 1.0; for (int i = 2; i <= n; ++i) r *= i; return r; };
  auto bin = [](int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
  };
  for (int i = 0; i < C2S_L * C2S_M * C2S_C; ++i) c[i] = 0.0;
  for (int l = 0; l < C2S_L; ++l) {
    const int nc = ncart(l);
    if (l <= 1) {
      for (int i = 0; i < nc; ++i) c[(l * C2S_M + i) * C2S_C + i] = 1.0;
      continue;
    }
    const double scale = std::sqrt((2 * l + 1) / (4.0 * M_PI));
    for (int m = -l; m <= l; ++m) {
      const int am = m < 0 ? -m : m;
      const double norm = 1.0 / (std::pow(2.0, am) * fact(l)) *
                          std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
      const int twovm = m < 0 ? 1 : 0;
      for (int t = 0; t <= (l - am) / 2; ++t)
        for (int u = 0; u <= t; ++u)
          for (int twov = twovm; twov <= am; twov += 2) {
            const int sg = t + (twov - twovm) / 2;
            const double coef = (sg % 2 ? -1.0 : 1.0) * std::pow(0.25, t) * bin(l, t) *
                                bin(l - t, am + t) * bin(t, u) * bin(am, twov);
            // powers (2t + am - 2u - twov, py, pz); the cartesian index needs
            // only py and pz
            const int py = 2 * u + twov, pz = l - 2 * t - am;
            const int k = (py + pz) * (py + pz + 1) / 2 + pz;
            c[(l * C2S_M + (m + l)) * C2S_C + k] += norm * scale * coef;
          }
    }
  }
}

ClassEntry g_classes[NCLASS];

const ClassEntry *class_table() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static bool filled = false;
  static bool ready[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    set_error("ERI kernel table: no usable current device");
    return nullptr;
  }
  std::lock_guard<std::mutex> g(mu);
  if (ready[dev]) return g_classes;
  double h[C2S_L * C2S_M * C2S_C];
  fill_c2s(h);
  ClassEntry *t = filled ? nullptr : g_classes;
  cudaError_t e = cudaSuccess;
  for (auto reg : {eri_register_bra0, eri_register_bra1, eri_register_bra2, eri_register_bra3,
                   eri_register_bra4, eri_register_bra5})
    if (e == cudaSuccess) e = reg(t, h);
  if (e == cudaSuccess) e = eri_register_gen(h);
  if (e == cudaSuccess && !filled) {
    // the f classes: k_eri_gen with run-time class sizes
    for (int li = 0; li <= ERI_LMAX; ++li)
      for (int lj = 0; lj <= li; ++lj)
        for (int lk = 0; lk <= ERI_LMAX; ++lk)
          for (int ll = 0; ll <= lk; ++ll) {
            if (pair_index(lk, ll) > pair_index(li, lj) || li < 3) continue;
            ClassEntry &ce = g_classes[class_id(li, lj, lk, ll)];
            ce = ClassEntry{};
            ce.gen = 1;
            ce.g = gen_class(li, lj, lk, ll);
            ce.nr = ce.g.nr;
            ce.slots = 1;
            ce.smem[0] = gen_smem_bytes(ce.g, 0);
            ce.smem[1] = gen_smem_bytes(ce.g, 1);
          }
  }
  if (e == cudaSuccess) filled = true;
  for (int c = 0; c < NCLASS && e == cudaSuccess && filled; ++c)
    for (int m = 0; m < 3 && e == cudaSuccess; ++m)
      if (!g_classes[c].gen)
        e = cudaFuncSetAttribute(g_classes[c].fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)g_classes[c].smem[m]);
  for (int c = 0; c < NCLASS && e == cudaSuccess && filled; ++c)
    for (int m = 0; m < 2 && e == cudaSuccess; ++m)
      if (!g_classes[c].gen && g_classes[c].lp[m])
        e = cudaFuncSetAttribute(g_classes[c].lp[m], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)g_classes[c].lp_smem[m]);
  if (e != cudaSuccess) {
    char msg[160];
    snprintf(msg, sizeof msg, "ERI kernel table set-up on device %d failed: %s", dev,
             cudaGetErrorString(e));
    cudaGetLastError();
    set_error(msg);
    return nullptr;
  }
  ready[dev] = true;
  return g_classes;
}

const double *rys_table_device() {
  const double *p = nullptr;
  cudaGetSymbolAddress((void **)&p, RYS_TAB);
  return p;
}

// ---------------------------------------------------------------- driver
#define LRB_CK(x)                                        \
  do {                                                   \
    cudaError_t e_ = (x);                                \
    if (e_ != cudaSuccess) {                             \
      set_error(cudaGetErrorString(e_));                 \
      return LRB_ERR_CUDA;                               \
    }                                                    \
  } while (0)

int eri_centers(const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                long long nenv, double *centers, int *d_err, cudaStream_t st) {
  const int T = 256;
  int herr = 0;
  LRB_CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  k_centers<<<(nbas + T - 1) / T, T, 0, st>>>(d_atm, natm, d_bas, nbas, d_env, nenv, centers, d_err);
  LRB_CK(cudaGetLastError());
  ++engine().launches;
  LRB_CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaStreamSynchronize(st));
  if (herr) return set_error("atm/bas/env index out of range"), LRB_ERR_INPUT;
  return LRB_OK;
}

void eri_centers_async(const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                       long long nenv, double *centers, int *d_err, cudaStream_t st) {
  if (nbas <= 0) return;
  const int T = 256;
  k_centers<<<(nbas + T - 1) / T, T, 0, st>>>(d_atm, natm, d_bas, nbas, d_env, nenv, centers, d_err);
  ++engine().launches;
}

int eri_batch_device(Engine &eng, double *out, int coord, const int *d_shls, long long nq,
                     const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                     long long nenv, cudaStream_t st, EriBatchStats *stats,
                     const double *centers_ready, int gc_screen) {
  if (nq <= 0) return LRB_OK;
  if (coord != 0 && coord != 1) return set_error("coord must be 0 or 1"), LRB_ERR_INPUT;
  const ClassEntry *tab = class_table();
  if (!tab) return LRB_ERR_CUDA;
  // workspace
  Workspace &w = eng.ws;
  const size_t q = (size_t)nq;
  char *base = w.reserve(st, q * sizeof(QuartetJob) * 2 + q * (4 * sizeof(unsigned) + 4 * sizeof(int)) +
                             q * 2 * sizeof(long long) + q * 4 * sizeof(int) + (size_t)nbas * 24 + 4096 +
                             (1 << 20));
  if (!base) return set_error("workspace allocation failed"), LRB_ERR_ALLOC;
  Carver cv(base);
  QuartetJob *jobs = cv.take<QuartetJob>(q);
  unsigned *keys = cv.take<unsigned>(q), *keys2 = cv.take<unsigned>(q);
  int *idx = cv.take<int>(q), *idx2 = cv.take<int>(q);
  long long *blk = cv.take<long long>(q), *out_off = cv.take<long long>(q);
  int *npair = cv.take<int>(2 * q), *pair_off = cv.take<int>(2 * q);
  double *centers = cv.take<double>(3 * (size_t)nbas);
  int *counters = cv.take<int>(NCLASS * 2 + 2);
  int *err = counters + NCLASS * 2;
  long long *starts = cv.take<long long>(NCLASS + 1);
  LRB_CK(cudaMemsetAsync(counters, 0, sizeof(int) * (NCLASS * 2 + 2), st));

  const int T = 256;
  if (!centers_ready) {
    k_centers<<<(nbas + T - 1) / T, T, 0, st>>>(d_atm, natm, d_bas, nbas, d_env, nenv, centers, err);
    LRB_CK(cudaGetLastError());
    // a bad shell must not reach the classifier: it reads bas[] of every shell
    int herr0 = 0;
    LRB_CK(cudaMemcpyAsync(&herr0, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    LRB_CK(cudaStreamSynchronize(st));
    if (herr0) return set_error("atm/bas/env index out of range"), LRB_ERR_INPUT;
  }
  const double *cen = centers_ready ? centers_ready : centers;
  k_classify<<<(unsigned)((nq + T - 1) / T), T, 0, st>>>(d_shls, nq, d_bas, nbas, coord, jobs, keys,
                                                         idx, blk, npair, err);
  LRB_CK(cudaGetLastError());
  // scans and sort (CUB, temp storage from the second arena)
  size_t tmp1 = 0, tmp2 = 0, tmp3 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp1, blk, out_off, (int)nq, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tmp2, npair, pair_off, (int)(2 * nq), st);
  cub::DeviceRadixSort::SortPairs(nullptr, tmp3, keys, keys2, idx, idx2, (int)nq, 0, 32, st);
  const size_t tmpb = std::max(tmp1, std::max(tmp2, tmp3));
  void *tmp = w.reserve_aux(st, tmpb + 2 * sizeof(long long) + 2 * sizeof(int) + 64);
  if (!tmp) return set_error("workspace allocation failed"), LRB_ERR_ALLOC;
  LRB_CK(cub::DeviceScan::ExclusiveSum(tmp, tmp1, blk, out_off, (int)nq, st));
  LRB_CK(cub::DeviceScan::ExclusiveSum(tmp, tmp2, npair, pair_off, (int)(2 * nq), st));
  LRB_CK(cub::DeviceRadixSort::SortPairs(tmp, tmp3, keys, keys2, idx, idx2, (int)nq, 0, 32, st));
  k_offsets<<<(unsigned)((nq + T - 1) / T), T, 0, st>>>(jobs, nq, out_off, pair_off);
  eng.launches += centers_ready ? 2 : 3;   // k_centers, k_classify, k_offsets
  // totals and class boundaries back to the host (small copies)
  long long last_blk = 0, last_off = 0;
  int last_np = 0, last_poff = 0, herr = 0;
  LRB_CK(cudaMemcpyAsync(&last_blk, blk + nq - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaMemcpyAsync(&last_off, out_off + nq - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaMemcpyAsync(&last_np, npair + 2 * nq - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaMemcpyAsync(&last_poff, pair_off + 2 * nq - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  k_class_starts<<<1, 64, 0, st>>>(keys2, nq, starts);
  ++eng.launches;
  long long cls_begin[NCLASS + 1];
  LRB_CK(cudaMemcpyAsync(cls_begin, starts, sizeof(long long) * (NCLASS + 1), cudaMemcpyDeviceToHost, st));
  // env[0] (screening cutoff) and env[8] (range-separation omega)
  double henv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  LRB_CK(cudaMemcpyAsync(henv, d_env, sizeof(double) * (size_t)std::min(nenv, 9LL),
                         cudaMemcpyDeviceToHost, st));
  LRB_CK(cudaStreamSynchronize(st));
  if (herr == 2) return set_error("shell index out of range"), LRB_ERR_INPUT;
  if (herr) return set_error("shell with l > 3, nprim > 31 or nctr != 1"), LRB_ERR_UNSUPPORTED;
  const long long npp = (long long)last_poff + last_np;
  if (npp > 2147483647LL) return set_error("too many primitive pairs in one batch"), LRB_ERR_INPUT;
  // pairs in natural order go to the second half, sorted ones to the first
  PrimPair *pp = (PrimPair *)w.reserve_pairs(st, 2 * (size_t)std::max(npp, 1LL) * sizeof(PrimPair));
  if (!pp) return set_error("workspace allocation failed"), LRB_ERR_ALLOC;
  if (npp > 0) {
    k_pairs_block<<<(unsigned)((2 * nq + PB_PAIRS - 1) / PB_PAIRS), PB_THREADS, 0, st>>>(
        jobs, nq, npair, pair_off, d_atm, d_bas, d_env, pp, pp + npp, gc_screen);
    ++eng.launches;
  }
  LRB_CK(cudaGetLastError());
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const double *rys = rys_table_device();
  EriParams prm;
  prm.jobs = jobs;
  prm.pp = pp;
  prm.centers = cen;
  prm.out = out;
  prm.expcutoff = henv[0] == 0.0 ? eng.expcutoff : std::max(40.0, henv[0]) + 1.0;
  prm.omega = henv[8];
  prm.sph = coord;
  for (int c = 0; c < NCLASS; ++c) {
    const long long end = cls_begin[c + 1];
    if (end <= cls_begin[c]) continue;
    const ClassEntry &ce = tab[c];
    prm.order = idx2 + cls_begin[c];
    prm.njobs = (int)(end - cls_begin[c]);
    int per_sm = 0;
    if (ce.gen)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gen_kernel(0), GEN_THREADS, ce.smem[0]);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ce.fn[0], ERI_THREADS, ce.smem[0]);
    if (per_sm < 1) per_sm = 1;
    const long long tasks = (prm.njobs + ce.slots - 1) / ce.slots;
    long long grid = (long long)nsm * per_sm;
    const long long need = ce.gen ? tasks : (tasks + ERI_WARPS - 1) / ERI_WARPS;
    if (grid > need) grid = need;
    ProfRecord rec{c, nullptr, nullptr};
    if (eng.profile) {
      cudaEventCreate(&rec.start);
      cudaEventCreate(&rec.stop);
      cudaEventRecord(rec.start, st);
    }
    FockParams nofock{};
    if (ce.gen)
      gen_kernel(0)<<<(unsigned)grid, GEN_THREADS, ce.smem[0], st>>>(prm, nofock, ce.g,
                                                                     rys + RYS_TAB_OFFSET[ce.nr],
                                                                     counters + c);
    else
      ce.fn[0]<<<(unsigned)grid, ERI_THREADS, ce.smem[0], st>>>(prm, nofock,
                                                                rys + RYS_TAB_OFFSET[ce.nr],
                                                                counters + c);
    LRB_CK(cudaGetLastError());
    ++eng.launches;
    if (eng.profile) {
      cudaEventRecord(rec.stop, st);
      eng.prof.push_back(rec);
    }
  }
  if (stats) {
    stats->nq = nq;
    stats->out_len = last_off + last_blk;
    stats->prim_pairs = npp;
  }
  return LRB_OK;
}

long long eri_batch_out_len(int coord, const int *shls, long long nq, const int *bas) {
  long long n = 0;
  for (long long q = 0; q < nq; ++q) {
    long long b = 1;
    for (int a = 0; a < 4; ++a) {
      const int *bs = bas + 8 * shls[4 * q + a];
      const int l = bs[1], nctr = bs[3] > 1 ? bs[3] : 1;   // contractions are rows too
      b *= (long long)(coord == 0 ? ncart(l) : nsph(l)) * nctr;
    }
    n += b;
  }
  return n;
}

}  // namespace lrb
