// Frozen-density gradient of the RHF energy with respect to basis exponents
// and contraction coefficients, env[s1:s2] (reference src/dscf.rs:320-565,
// src/utils.rs:152-175):
//   dH = sum P (dT + dV),  dR = d/dtheta 1/2 sum (P P - 1/2 P P)(ij|kl),
//   dS = sum Q dS with Q = P F P,  danalytical = dH + dR - dS/2.
// The reference obtains each part by Enzyme reverse passes; here dR comes from
// the adjoint ERI kernel (grad_kernel.cuh) and dH, dS from a one-electron
// derivative kernel, all contracted with the densities on the GPU.
#include <cublas_v2.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

const double *rys_table_device();
int scf_dense_fock(MolCtx &m, const double *P, double *F, cudaStream_t st);

#define GR_CK(x)                                  \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) {                      \
      set_error(cudaGetErrorString(e_));          \
      return LRB_ERR_CUDA;                        \
    }                                             \
  } while (0)

GradEntry g_grad_classes[NGRADCLS][NGRADMODE];

// Kernel pointers and shared-memory sizes are filled once per process; the
// large-shared-memory attribute is per device and set for each device used.
// The adjoint kernels cover shells up to d.
static int grad_shells_supported(const MolCtx &m) {
  if (m.gc) return set_error("gradients: generally contracted shells are not supported"),
            LRB_ERR_UNSUPPORTED;
  if (m.nenv > 8 && m.h_env[8] != 0.0)
    return set_error("gradients: range-separated integrals (env[8] != 0) are not supported"),
           LRB_ERR_UNSUPPORTED;
  for (int s = 0; s < m.nbas; ++s)
    if (m.h_bas[8 * s + 1] > 2)
      return set_error("gradients: shells up to l = 2 are supported"), LRB_ERR_UNSUPPORTED;
  return LRB_OK;
}

static int grad_table_init() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static bool filled = false;
  static bool ready[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return set_error("gradient kernel table: no usable current device"), LRB_ERR_CUDA;
  }
  std::lock_guard<std::mutex> g(mu);
  if (ready[dev]) return LRB_OK;
  if (!filled) {
    GradEntry *t = &g_grad_classes[0][0];
    for (int i = 0; i < NGRADCLS * NGRADMODE; ++i) t[i] = GradEntry{nullptr, 0, 1, 1};
    grad_register_x0(t);
    grad_register_x1(t);
    grad_register_x2(t);
    grad_register_n0(t);
    grad_register_n1(t);
    grad_register_n2(t);
    filled = true;
  }
  for (int c = 0; c < NGRADCLS; ++c)
    for (int r = 0; r < NGRADMODE; ++r)
      if (g_grad_classes[c][r].fn) {
        const cudaError_t e = cudaFuncSetAttribute(g_grad_classes[c][r].fn,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)g_grad_classes[c][r].smem);
        if (e != cudaSuccess) {
          cudaGetLastError();
          return set_error(cudaGetErrorString(e)), LRB_ERR_CUDA;
        }
      }
  ready[dev] = true;
  return LRB_OK;
}

namespace {

__device__ inline int pcls_of(int a, int b) { return a * (a + 1) / 2 + b; }

// canonical pair pairs (b >= k) -> four jobs (one per differentiated shell)
__global__ void k_grad_jobs(const PairInfo *__restrict__ pairs, const double *__restrict__ Q,
                            const double *__restrict__ Dsh, const int *__restrict__ bas, int nbas,
                            long long ncand, double tau, GradJob *jobs, unsigned *keys, int *idx,
                            unsigned long long *count, unsigned long long cap) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ncand) return;
  int b = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)b * (b + 1) / 2 > t) --b;
  while ((long long)(b + 1) * (b + 2) / 2 <= t) ++b;
  const int k = (int)(t - (long long)b * (b + 1) / 2);
  const PairInfo pb = pairs[b], pk = pairs[k];
  const int I = pb.ish, J = pb.jsh, K = pk.ish, L = pk.jsh;
  const double d = fmax(fmax(2.0 * Dsh[I * nbas + J], 2.0 * Dsh[K * nbas + L]),
                        fmax(fmax(Dsh[I * nbas + K], Dsh[I * nbas + L]),
                             fmax(Dsh[J * nbas + K], Dsh[J * nbas + L])));
  if (Q[b] * Q[k] * d < tau) return;
  const unsigned long long base = atomicAdd(count, 4ull);
  if (base + 4 > cap) return;
  for (int v = 0; v < 4; ++v) {
    const int bp = v < 2 ? b : k, kp = v < 2 ? k : b;
    const int xs = v & 1;
    const PairInfo pX = pairs[bp], pO = pairs[kp];
    const int X = xs ? pX.jsh : pX.ish, Y = xs ? pX.ish : pX.jsh;
    const int lx = bas[8 * X + 1], ly = bas[8 * Y + 1];
    const int cls = (lx * 3 + ly) * 6 + pcls_of(bas[8 * pO.ish + 1], bas[8 * pO.jsh + 1]);
    const int kprod = pX.npp * pO.npp;
    GradJob j;
    j.bp = bp; j.kp = kp; j.xsecond = xs; j.pad = 0;
    jobs[base + v] = j;
    keys[base + v] = ((unsigned)cls << 20) | (unsigned)(0xfffff - kprod);
    idx[base + v] = (int)(base + v);
  }
}

__global__ void k_grad_starts(const unsigned *__restrict__ keys, long long n, long long *starts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > NGRADCLS) return;
  long long lo = 0, hi = n;
  const unsigned key = (unsigned)c << 20;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  starts[c] = lo;
}

__device__ __forceinline__ double fac_sp(int l) {
  return l == 0 ? 0.28209479177387814 : (l == 1 ? 0.48860251190291992 : 1.0);
}
__device__ __forceinline__ void cart_of(int l, int n, int &x, int &y, int &z) {
  int t = 0;
  while ((t + 1) * (t + 2) / 2 <= n) ++t;
  z = n - t * (t + 1) / 2;
  y = t - z;
  x = l - t;
}
__device__ double os1(int ti, int tj, double xpa, double xpb, double oo2p) {
  double s[7][7];
  for (int i = 0; i <= ti; ++i)
    for (int j = 0; j <= tj; ++j) {
      double v;
      if (i == 0 && j == 0) v = 1.0;
      else if (i > 0) {
        v = xpa * s[i - 1][j];
        if (i > 1) v += oo2p * (i - 1) * s[i - 2][j];
        if (j > 0) v += oo2p * j * s[i - 1][j - 1];
      } else {
        v = xpb * s[0][j - 1];
        if (j > 1) v += oo2p * (j - 1) * s[0][j - 2];
      }
      s[i][j] = v;
    }
  return s[ti][tj];
}

// Primitive integral of the operator (0 S, 1 T, 2 V) between cartesian
// monomials ia (on A, exponent ai) and jb (on B, exponent bj), without the
// contraction coefficients; same conventions as int1e.cu.
__device__ double prim1e(int op, const int ia[3], const int jb[3], double ai, double bj,
                         const double *A, const double *B, int li, int lj, const int *atm,
                         int natm, const double *env, const double *rys, int cnuc = -1) {
  const double p = ai + bj;
  const double rab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                      (A[2] - B[2]) * (A[2] - B[2]);
  const double e = fac_sp(li) * fac_sp(lj) * exp(-ai * bj / p * rab2);
  double P[3];
  for (int d = 0; d < 3; ++d) P[d] = (ai * A[d] + bj * B[d]) / p;
  if (op <= 1) {
    const double pre = e * pow(M_PI / p, 1.5);
    double s1[3];
    for (int d = 0; d < 3; ++d) s1[d] = os1(ia[d], jb[d], P[d] - A[d], P[d] - B[d], 0.5 / p);
    if (op == 0) return pre * s1[0] * s1[1] * s1[2];
    double v = 0.0;
    for (int d = 0; d < 3; ++d) {
      const int j = jb[d];
      double tt = -2.0 * bj * (2 * j + 1) * s1[d] +
                  4.0 * bj * bj * os1(ia[d], j + 2, P[d] - A[d], P[d] - B[d], 0.5 / p);
      if (j >= 2) tt += j * (j - 1) * os1(ia[d], j - 2, P[d] - A[d], P[d] - B[d], 0.5 / p);
      tt *= -0.5;
      double o = 1.0;
      for (int k = 0; k < 3; ++k)
        if (k != d) o *= s1[k];
      v += tt * o;
    }
    return pre * v;
  }
  const int tot = ia[0] + ia[1] + ia[2] + jb[0] + jb[1] + jb[2];
  const int nr = tot / 2 + 1;
  double acc = 0.0;
  // all nuclei, or only nucleus cnuc
  for (int c = cnuc < 0 ? 0 : cnuc; c < (cnuc < 0 ? natm : cnuc + 1); ++c) {
    const double *C = env + atm[6 * c + 1];
    const double z = -fabs((double)atm[6 * c]);
    const double x = p * ((P[0] - C[0]) * (P[0] - C[0]) + (P[1] - C[1]) * (P[1] - C[1]) +
                          (P[2] - C[2]) * (P[2] - C[2]));
    double u[5], w[5];
    for (int f = 0; f < 2 * nr; ++f) {
      double v;
      switch (nr) {
        case 1: v = rys_function<1>(rys + rys_tab_offset(1), x, f); break;
        case 2: v = rys_function<2>(rys + rys_tab_offset(2), x, f); break;
        case 3: v = rys_function<3>(rys + rys_tab_offset(3), x, f); break;
        case 4: v = rys_function<4>(rys + rys_tab_offset(4), x, f); break;
        default: v = rys_function<5>(rys + rys_tab_offset(5), x, f); break;
      }
      if (f < nr) u[f] = v; else w[f - nr] = v;
    }
    const double pre = e * 2.0 * M_PI / p * z;
    for (int r = 0; r < nr; ++r) {
      const double t2 = u[r] / (1.0 + u[r]);
      double prod = 1.0;
      for (int d = 0; d < 3; ++d) {
        double g[11];
        g[0] = 1.0;
        const double c0 = (P[d] - A[d]) - t2 * (P[d] - C[d]);
        const double b1 = 0.5 / p * (1.0 - t2);
        const int top = ia[d] + jb[d];
        if (top > 0) g[1] = c0;
        for (int k = 1; k < top; ++k) g[k + 1] = c0 * g[k] + k * b1 * g[k - 1];
        const double ab = A[d] - B[d];
        double v = 0.0, binc = 1.0, pw = 1.0;
        for (int k = jb[d]; k >= 0; --k) {
          v += binc * pw * g[ia[d] + k];
          pw *= ab;
          binc = binc * k / (jb[d] - k + 1);
        }
        prod *= v;
      }
      acc += pre * w[r] * prod;
    }
  }
  return acc;
}

// One thread per ordered AO pair (mu, nu): bra-side derivatives of
// W[mu nu] M[mu nu] for every primitive of mu's shell, times 2 (the ket side
// gives the same by symmetry of W and M).
__global__ void k_grad1e(int op, double scale, int n, const int *__restrict__ ao_shell,
                         const int *__restrict__ ao_comp, const int *__restrict__ atm, int natm,
                         const int *__restrict__ bas, const double *__restrict__ env,
                         const double *__restrict__ W, const double *__restrict__ rys, int s1,
                         double *grad) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int mu = (int)(t / n), nu = (int)(t % n);
  const double wmn = W[t] * 2.0 * scale;
  if (wmn == 0.0) return;
  const int si = ao_shell[mu], sj = ao_shell[nu];
  const int *bi = bas + 8 * si, *bj = bas + 8 * sj;
  const int li = bi[1], lj = bj[1];
  int ia[3], jb[3];
  cart_of(li, ao_comp[mu], ia[0], ia[1], ia[2]);
  cart_of(lj, ao_comp[nu], jb[0], jb[1], jb[2]);
  const double *A = env + atm[6 * bi[0] + 1], *B = env + atm[6 * bj[0] + 1];
  for (int ip = 0; ip < bi[2]; ++ip) {
    const double ai = env[bi[5] + ip], cip = env[bi[6] + ip];
    double dcoef = 0.0, dexp = 0.0;
    for (int jp = 0; jp < bj[2]; ++jp) {
      const double bjx = env[bj[5] + jp], cj = env[bj[6] + jp];
      dcoef += cj * prim1e(op, ia, jb, ai, bjx, A, B, li, lj, atm, natm, env, rys);
      double r = 0.0;
      for (int d = 0; d < 3; ++d) {
        int ib[3] = {ia[0], ia[1], ia[2]};
        ib[d] += 2;
        r += prim1e(op, ib, jb, ai, bjx, A, B, li, lj, atm, natm, env, rys);
      }
      dexp -= cip * cj * r;
    }
    atomicAdd(&grad[bi[6] + ip - s1], wmn * dcoef);
    atomicAdd(&grad[bi[5] + ip - s1], wmn * dexp);
  }
}

// Nuclear-coordinate derivative of sum W[mu nu] O[mu nu], one thread per
// ordered AO pair: the bra function's centre derivative
//   d/dA_d (x^a e^{-p r^2}) = 2 p x^(a+e_d) e^.. - a_d x^(a-e_d) e^..
// times 2 (the ket side is the same by symmetry of W and O), added to the
// bra's atom.  For the nuclear attraction (op 2) each nucleus C also takes
// the Hellmann-Feynman term, which by translational invariance of the
// C-term is minus the sum of both basis-centre derivatives.
__global__ void k_grad1e_nuc(int op, double scale, int n, const int *__restrict__ ao_shell,
                             const int *__restrict__ ao_comp, const int *__restrict__ atm,
                             int natm, const int *__restrict__ bas, const double *__restrict__ env,
                             const double *__restrict__ W, const double *__restrict__ rys,
                             double *gatom) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int mu = (int)(t / n), nu = (int)(t % n);
  const double wmn = W[t] * 2.0 * scale;
  if (wmn == 0.0) return;
  const int si = ao_shell[mu], sj = ao_shell[nu];
  const int *bi = bas + 8 * si, *bj = bas + 8 * sj;
  const int li = bi[1], lj = bj[1];
  int ia[3], jb[3];
  cart_of(li, ao_comp[mu], ia[0], ia[1], ia[2]);
  cart_of(lj, ao_comp[nu], jb[0], jb[1], jb[2]);
  const double *A = env + atm[6 * bi[0] + 1], *B = env + atm[6 * bj[0] + 1];
  const int na = op == 2 ? natm : 1;
  for (int c = 0; c < na; ++c) {
    const int cn = op == 2 ? c : -1;
    double g[3] = {0.0, 0.0, 0.0};
    for (int ip = 0; ip < bi[2]; ++ip) {
      const double ai = env[bi[5] + ip], cip = env[bi[6] + ip];
      for (int jp = 0; jp < bj[2]; ++jp) {
        const double bjx = env[bj[5] + jp], cc = cip * env[bj[6] + jp];
        for (int d = 0; d < 3; ++d) {
          int ib[3] = {ia[0], ia[1], ia[2]};
          ib[d] += 1;
          double v = 2.0 * ai * prim1e(op, ib, jb, ai, bjx, A, B, li, lj, atm, natm, env, rys, cn);
          if (ia[d] > 0) {
            ib[d] -= 2;
            v -= ia[d] * prim1e(op, ib, jb, ai, bjx, A, B, li, lj, atm, natm, env, rys, cn);
          }
          g[d] += cc * v;
        }
      }
    }
    for (int d = 0; d < 3; ++d) {
      atomicAdd(&gatom[3 * bi[0] + d], wmn * g[d]);
      if (op == 2) atomicAdd(&gatom[3 * c + d], -wmn * g[d]);
    }
  }
}

// Overlap Jacobian with respect to env[s1:s1+L] (the reference's dS_u,
// src/dscf.rs:96-151): one thread per AO pair (mu, nu) owns the row
// out[(nu * n + mu) * L + l] = d S[mu, nu] / d env[s1 + l].  Bra-side
// parameters are those of mu's shell, ket-side those of nu's (the two add
// when shells share parameters); coefficients c_p and exponents a_p as in
// k_grad1e.
__global__ void k_dS_u(int n, int L, int s1, const int *__restrict__ ao_shell,
                       const int *__restrict__ ao_comp, const int *__restrict__ atm, int natm,
                       const int *__restrict__ bas, const double *__restrict__ env,
                       const double *__restrict__ rys, double *out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int mu = (int)(t / n), nu = (int)(t % n);
  double *row = out + ((long long)nu * n + mu) * L;
  for (int side = 0; side < 2; ++side) {
    const int a = side == 0 ? mu : nu, b = side == 0 ? nu : mu;   // a carries the parameters
    const int sa = ao_shell[a], sb = ao_shell[b];
    const int *ba = bas + 8 * sa, *bb = bas + 8 * sb;
    int ia[3], jb[3];
    cart_of(ba[1], ao_comp[a], ia[0], ia[1], ia[2]);
    cart_of(bb[1], ao_comp[b], jb[0], jb[1], jb[2]);
    const double *A = env + atm[6 * ba[0] + 1], *B = env + atm[6 * bb[0] + 1];
    for (int ip = 0; ip < ba[2]; ++ip) {
      const double ai = env[ba[5] + ip], cip = env[ba[6] + ip];
      double dcoef = 0.0, dexp = 0.0;
      for (int jp = 0; jp < bb[2]; ++jp) {
        const double bj = env[bb[5] + jp], cj = env[bb[6] + jp];
        dcoef += cj * prim1e(0, ia, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
        double r = 0.0;
        for (int d = 0; d < 3; ++d) {
          int ib[3] = {ia[0], ia[1], ia[2]};
          ib[d] += 2;
          r += prim1e(0, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
        }
        dexp -= cip * cj * r;
      }
      const int kc = ba[6] + ip - s1, ke = ba[5] + ip - s1;
      if (kc >= 0 && kc < L) row[kc] += dcoef;
      if (ke >= 0 && ke < L) row[ke] += dexp;
    }
  }
}

// Full Jacobian of a one-electron matrix (op 0 S, 1 T, 2 V) with respect to
// every env entry: row (nu * n + mu) holds d O[mu, nu] / d env[l] for all l
// (the layout of the reference's Enzyme checks, checks/overlap.rs:96-175).
// Columns: exponents and coefficients of the two shells, the coordinates of
// the two atoms (centre derivatives 2 a x^(a+e_d) - a_d x^(a-e_d)) and, for
// V, every nucleus position (Hellmann-Feynman term, minus the two centre
// derivatives of that nucleus's term).  One thread per AO pair.
__global__ void k_d1e_env(int op, int n, long long nenv, const int *__restrict__ ao_shell,
                          const int *__restrict__ ao_comp, const int *__restrict__ atm, int natm,
                          const int *__restrict__ bas, const double *__restrict__ env,
                          const double *__restrict__ rys, double *out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int mu = (int)(t / n), nu = (int)(t % n);
  double *row = out + ((long long)nu * n + mu) * nenv;
  for (int side = 0; side < 2; ++side) {
    const int a = side == 0 ? mu : nu, b = side == 0 ? nu : mu;   // a is differentiated
    const int sa = ao_shell[a], sb = ao_shell[b];
    const int *ba = bas + 8 * sa, *bb = bas + 8 * sb;
    int ia[3], jb[3];
    cart_of(ba[1], ao_comp[a], ia[0], ia[1], ia[2]);
    cart_of(bb[1], ao_comp[b], jb[0], jb[1], jb[2]);
    const double *A = env + atm[6 * ba[0] + 1], *B = env + atm[6 * bb[0] + 1];
    const int pa = atm[6 * ba[0] + 1];
    for (int ip = 0; ip < ba[2]; ++ip) {
      const double ai = env[ba[5] + ip], cip = env[ba[6] + ip];
      double dcoef = 0.0, dexp = 0.0, dc[3] = {0.0, 0.0, 0.0};
      for (int jp = 0; jp < bb[2]; ++jp) {
        const double bj = env[bb[5] + jp], cj = env[bb[6] + jp];
        dcoef += cj * prim1e(op, ia, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
        double r = 0.0;
        for (int d = 0; d < 3; ++d) {
          int ib[3] = {ia[0], ia[1], ia[2]};
          ib[d] += 2;
          r += prim1e(op, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
          ib[d] -= 1;
          double v = 2.0 * ai * prim1e(op, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
          if (ia[d] > 0) {
            ib[d] -= 2;
            v -= ia[d] * prim1e(op, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys);
          }
          dc[d] += cip * cj * v;
        }
        dexp -= cip * cj * r;
      }
      row[ba[6] + ip] += dcoef;
      row[ba[5] + ip] += dexp;
      for (int d = 0; d < 3; ++d) row[pa + d] += dc[d];
    }
    if (op == 2) {
      for (int c = 0; c < natm; ++c) {
        double g[3] = {0.0, 0.0, 0.0};
        for (int ip = 0; ip < ba[2]; ++ip) {
          const double ai = env[ba[5] + ip], cip = env[ba[6] + ip];
          for (int jp = 0; jp < bb[2]; ++jp) {
            const double bj = env[bb[5] + jp], cc = cip * env[bb[6] + jp];
            for (int d = 0; d < 3; ++d) {
              int ib[3] = {ia[0], ia[1], ia[2]};
              ib[d] += 1;
              double v = 2.0 * ai * prim1e(op, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys, c);
              if (ia[d] > 0) {
                ib[d] -= 2;
                v -= ia[d] * prim1e(op, ib, jb, ai, bj, A, B, ba[1], bb[1], atm, natm, env, rys, c);
              }
              g[d] += cc * v;
            }
          }
        }
        const int pc = atm[6 * c + 1];
        for (int d = 0; d < 3; ++d) row[pc + d] -= g[d];
      }
    }
  }
}

// d/dR of the nuclear repulsion, one thread per atom.
__global__ void k_grad_nn(const int *__restrict__ atm, int natm, const double *__restrict__ env,
                          double *gatom) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natm) return;
  const double *Ra = env + atm[6 * a + 1];
  const double za = (double)atm[6 * a];
  double g[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < natm; ++b) {
    if (b == a) continue;
    const double *Rb = env + atm[6 * b + 1];
    const double d[3] = {Ra[0] - Rb[0], Ra[1] - Rb[1], Ra[2] - Rb[2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double f = -za * (double)atm[6 * b] / (r2 * sqrt(r2));
    for (int k = 0; k < 3; ++k) g[k] += f * d[k];
  }
  for (int k = 0; k < 3; ++k) gatom[3 * a + k] += g[k];
}

}  // namespace

// Adjoint ERI pass over all canonical quartets that survive Schwarz x density
// screening (density Ps, already scaled), launching mode slots
// [slot0, slot0 + nslot) of the class table with the parameters in gp.
static int grad_eri_pass(MolCtx &m, const double *Ps, double tau, int slot0, int nslot,
                         GradParams gp, cudaStream_t st) {
  Engine &eng = engine();
  const int nbas = m.nbas;
  const double *rys = rys_table_device();
  const long long ncand = (long long)m.npairs * (m.npairs + 1) / 2;
  const size_t cap = (size_t)ncand * 4;
  GradJob *jobs = nullptr;
  unsigned *keys = nullptr, *keys2 = nullptr;
  int *idx = nullptr, *idx2 = nullptr, *counters = nullptr;
  unsigned long long *count = nullptr;
  long long *starts = nullptr;
  GR_CK(cudaMallocAsync((void **)&jobs, sizeof(GradJob) * cap, st));
  GR_CK(cudaMallocAsync((void **)&keys, sizeof(unsigned) * cap, st));
  GR_CK(cudaMallocAsync((void **)&keys2, sizeof(unsigned) * cap, st));
  GR_CK(cudaMallocAsync((void **)&idx, sizeof(int) * cap, st));
  GR_CK(cudaMallocAsync((void **)&idx2, sizeof(int) * cap, st));
  GR_CK(cudaMallocAsync((void **)&counters, sizeof(int) * NGRADMODE * NGRADCLS, st));
  GR_CK(cudaMallocAsync((void **)&count, sizeof(unsigned long long), st));
  GR_CK(cudaMallocAsync((void **)&starts, sizeof(long long) * (NGRADCLS + 1), st));
  GR_CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
  GR_CK(cudaMemsetAsync(counters, 0, sizeof(int) * NGRADMODE * NGRADCLS, st));
  dens_max_device(m, Ps, st);
  k_grad_jobs<<<(unsigned)((ncand + 255) / 256), 256, 0, st>>>(m.pairs, m.Q, m.Dsh, m.bas, nbas, ncand,
                                                               tau, jobs, keys, idx, count, cap);
  eng.launches += 2;
  unsigned long long nj = 0;
  GR_CK(cudaMemcpyAsync(&nj, count, sizeof(nj), cudaMemcpyDeviceToHost, st));
  GR_CK(cudaStreamSynchronize(st));
  if (nj > cap) nj = cap;
  void *tmp = nullptr;
  if (nj > 0) {
    size_t tmpb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys, keys2, idx, idx2, (int)nj, 0, 32, st);
    GR_CK(cudaMallocAsync(&tmp, tmpb + 16, st));
    GR_CK(cub::DeviceRadixSort::SortPairs(tmp, tmpb, keys, keys2, idx, idx2, (int)nj, 0, 32, st));
    k_grad_starts<<<1, 64, 0, st>>>(keys2, (long long)nj, starts);
    eng.launches++;
    long long cb[NGRADCLS + 1];
    GR_CK(cudaMemcpyAsync(cb, starts, sizeof(cb), cudaMemcpyDeviceToHost, st));
    GR_CK(cudaStreamSynchronize(st));
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    gp.jobs = jobs;
    for (int c = 0; c < NGRADCLS; ++c) {
      if (cb[c + 1] <= cb[c]) continue;
      gp.order = idx2 + cb[c];
      gp.njobs = (int)(cb[c + 1] - cb[c]);
      for (int r = slot0; r < slot0 + nslot; ++r) {
        const GradEntry &ge = g_grad_classes[c][r];
        if (!ge.fn) continue;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ge.fn, GRAD_THREADS, ge.smem);
        if (per_sm < 1) per_sm = 1;
        const long long tasks = (gp.njobs + ge.slots - 1) / ge.slots;
        long long grid = (long long)nsm * per_sm;
        const long long needg = (tasks + GRAD_WARPS - 1) / GRAD_WARPS;
        if (grid > needg) grid = needg;
        ge.fn<<<(unsigned)grid, GRAD_THREADS, ge.smem, st>>>(gp, rys + RYS_TAB_OFFSET[ge.nr],
                                                             counters + NGRADMODE * c + r);
        GR_CK(cudaGetLastError());
        eng.launches++;
      }
    }
  }
  for (void *p : {(void *)jobs, (void *)keys, (void *)keys2, (void *)idx, (void *)idx2,
                  (void *)counters, (void *)count, (void *)starts, tmp})
    if (p) cudaFreeAsync(p, st);
  return LRB_OK;
}

int grad_run(MolCtx &m, const double *d_P, double cH, double cR, double cS, double tau,
             double *d_grad, int s1, cudaStream_t st) {
  if (int rc0 = grad_shells_supported(m)) return rc0;
  if (int rc0 = grad_table_init()) return rc0;
  Engine &eng = engine();
  const int n = m.nao, nbas = m.nbas;
  const long long nn = (long long)n * n;
  const double *rys = rys_table_device();
  // AO maps
  std::vector<int> ao_shell, ao_comp;
  for (int s = 0; s < nbas; ++s)
    for (int c = 0; c < ncart(m.h_bas[8 * s + 1]); ++c) { ao_shell.push_back(s); ao_comp.push_back(c); }
  int *d_map = nullptr;
  GR_CK(cudaMallocAsync((void **)&d_map, sizeof(int) * 2 * n, st));
  GR_CK(cudaMemcpyAsync(d_map, ao_shell.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemcpyAsync(d_map + n, ao_comp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  const unsigned gb = (unsigned)((nn + 127) / 128);
  if (cH != 0.0) {
    k_grad1e<<<gb, 128, 0, st>>>(1, cH, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, d_P, rys,
                                 s1, d_grad);
    k_grad1e<<<gb, 128, 0, st>>>(2, cH, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, d_P, rys,
                                 s1, d_grad);
    eng.launches += 2;
  }
  if (cS != 0.0) {
    // Q = P F P with F = H + G(P)
    double *F = nullptr, *Qm = nullptr, *Wk = nullptr;
    GR_CK(cudaMallocAsync((void **)&F, sizeof(double) * nn, st));
    GR_CK(cudaMallocAsync((void **)&Qm, sizeof(double) * nn, st));
    GR_CK(cudaMallocAsync((void **)&Wk, sizeof(double) * nn, st));
    int rc = scf_dense_fock(m, d_P, F, st);
    if (rc) return rc;
    cublasHandle_t h = grad_blas();
    cublasSetStream(h, st);
    const double one = 1.0, zero = 0.0;
    cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, d_P, n, F, n, &zero, Wk, n);
    cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, Wk, n, d_P, n, &zero, Qm, n);
    k_grad1e<<<gb, 128, 0, st>>>(0, cS, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, Qm, rys,
                                 s1, d_grad);
    eng.launches++;
    cudaFreeAsync(F, st);
    cudaFreeAsync(Qm, st);
    cudaFreeAsync(Wk, st);
  }
  if (cR != 0.0) {
    // scale the density so the adjoint kernels accumulate cR * dR
    double *Ps = nullptr;
    GR_CK(cudaMallocAsync((void **)&Ps, sizeof(double) * nn, st));
    GR_CK(cudaMemcpyAsync(Ps, d_P, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    // Gamma is quadratic in P: scale P by sqrt(|cR|) (sign handled below)
    const double sc = std::sqrt(std::fabs(cR));
    cublasHandle_t h = grad_blas();
    cublasSetStream(h, st);
    cublasDscal(h, (int)nn, &sc, Ps, 1);
    const size_t glen = (size_t)(m.nenv - s1);
    double *gR = nullptr;
    GR_CK(cudaMallocAsync((void **)&gR, sizeof(double) * glen, st));
    GR_CK(cudaMemsetAsync(gR, 0, sizeof(double) * glen, st));
    GradParams gp{};
    gp.pairs = m.pairs; gp.pp = m.pp; gp.centers = m.centers;
    gp.bas = m.bas; gp.aooff = m.aooff; gp.env = m.env; gp.P = Ps; gp.n = n;
    gp.expcutoff = eng.expcutoff; gp.grad = gR; gp.s1 = s1; gp.gatom = nullptr;
    int rc = grad_eri_pass(m, Ps, tau, 0, 2, gp, st);
    if (rc) return rc;
    // d_grad += sign(cR) * gR
    const double sg = cR < 0 ? -1.0 : 1.0;
    cublasDaxpy(h, (int)glen, &sg, gR, 1, d_grad, 1);
    cudaFreeAsync(gR, st);
    cudaFreeAsync(Ps, st);
  }
  cudaFreeAsync(d_map, st);
  GR_CK(cudaStreamSynchronize(st));
  GR_CK(cudaGetLastError());
  return LRB_OK;
}

int dS_u_run(MolCtx &m, int s1, int L, double *d_out, cudaStream_t st) {
  if (int rc0 = grad_shells_supported(m)) return rc0;
  const int n = m.nao, nbas = m.nbas;
  const long long nn = (long long)n * n;
  std::vector<int> ao_shell, ao_comp;
  for (int s = 0; s < nbas; ++s)
    for (int c = 0; c < ncart(m.h_bas[8 * s + 1]); ++c) { ao_shell.push_back(s); ao_comp.push_back(c); }
  int *d_map = nullptr;
  GR_CK(cudaMallocAsync((void **)&d_map, sizeof(int) * 2 * n, st));
  GR_CK(cudaMemcpyAsync(d_map, ao_shell.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemcpyAsync(d_map + n, ao_comp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemsetAsync(d_out, 0, sizeof(double) * (size_t)nn * L, st));
  k_dS_u<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(n, L, s1, d_map, d_map + n, m.atm, m.natm,
                                                       m.bas, m.env, rys_table_device(), d_out);
  engine().launches++;
  cudaFreeAsync(d_map, st);
  GR_CK(cudaGetLastError());
  return LRB_OK;
}

int d1e_env_run(MolCtx &m, int op, double *d_out, cudaStream_t st) {
  if (int rc0 = grad_shells_supported(m)) return rc0;
  const int n = m.nao, nbas = m.nbas;
  const long long nn = (long long)n * n;
  std::vector<int> ao_shell, ao_comp;
  for (int s = 0; s < nbas; ++s)
    for (int c = 0; c < ncart(m.h_bas[8 * s + 1]); ++c) { ao_shell.push_back(s); ao_comp.push_back(c); }
  int *d_map = nullptr;
  GR_CK(cudaMallocAsync((void **)&d_map, sizeof(int) * 2 * n, st));
  GR_CK(cudaMemcpyAsync(d_map, ao_shell.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemcpyAsync(d_map + n, ao_comp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemsetAsync(d_out, 0, sizeof(double) * (size_t)nn * m.nenv, st));
  k_d1e_env<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(op, n, m.nenv, d_map, d_map + n, m.atm,
                                                          m.natm, m.bas, m.env, rys_table_device(),
                                                          d_out);
  engine().launches++;
  cudaFreeAsync(d_map, st);
  GR_CK(cudaGetLastError());
  return LRB_OK;
}

int grad_nuc_run(MolCtx &m, const double *d_P, double tau, double *d_gatom, cudaStream_t st) {
  if (int rc0 = grad_shells_supported(m)) return rc0;
  if (int rc0 = grad_table_init()) return rc0;
  Engine &eng = engine();
  const int n = m.nao, nbas = m.nbas;
  const long long nn = (long long)n * n;
  const double *rys = rys_table_device();
  std::vector<int> ao_shell, ao_comp;
  for (int s = 0; s < nbas; ++s)
    for (int c = 0; c < ncart(m.h_bas[8 * s + 1]); ++c) { ao_shell.push_back(s); ao_comp.push_back(c); }
  int *d_map = nullptr;
  double *F = nullptr, *Qm = nullptr, *Wk = nullptr;
  GR_CK(cudaMallocAsync((void **)&d_map, sizeof(int) * 2 * n, st));
  GR_CK(cudaMemcpyAsync(d_map, ao_shell.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  GR_CK(cudaMemcpyAsync(d_map + n, ao_comp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  const unsigned gb = (unsigned)((nn + 127) / 128);
  // dH: kinetic and nuclear attraction (with the Hellmann-Feynman term)
  k_grad1e_nuc<<<gb, 128, 0, st>>>(1, 1.0, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, d_P,
                                   rys, d_gatom);
  k_grad1e_nuc<<<gb, 128, 0, st>>>(2, 1.0, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, d_P,
                                   rys, d_gatom);
  // -1/2 sum (P F P) dS
  GR_CK(cudaMallocAsync((void **)&F, sizeof(double) * nn, st));
  GR_CK(cudaMallocAsync((void **)&Qm, sizeof(double) * nn, st));
  GR_CK(cudaMallocAsync((void **)&Wk, sizeof(double) * nn, st));
  int rc = scf_dense_fock(m, d_P, F, st);
  if (rc) return rc;
  cublasHandle_t h = grad_blas();
  cublasSetStream(h, st);
  const double one = 1.0, zero = 0.0;
  cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, d_P, n, F, n, &zero, Wk, n);
  cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, Wk, n, d_P, n, &zero, Qm, n);
  k_grad1e_nuc<<<gb, 128, 0, st>>>(0, -0.5, n, d_map, d_map + n, m.atm, m.natm, m.bas, m.env, Qm,
                                   rys, d_gatom);
  k_grad_nn<<<(m.natm + 127) / 128, 128, 0, st>>>(m.atm, m.natm, m.env, d_gatom);
  eng.launches += 4;
  // dR: centre derivatives of the ERIs contracted with Gamma
  GradParams gp{};
  gp.pairs = m.pairs; gp.pp = m.pp; gp.centers = m.centers;
  gp.bas = m.bas; gp.aooff = m.aooff; gp.env = m.env; gp.P = d_P; gp.n = n;
  gp.expcutoff = eng.expcutoff; gp.grad = nullptr; gp.s1 = 0; gp.gatom = d_gatom;
  rc = grad_eri_pass(m, d_P, tau, 2, 2, gp, st);
  if (rc) return rc;
  for (void *p : {(void *)F, (void *)Qm, (void *)Wk, (void *)d_map}) cudaFreeAsync(p, st);
  GR_CK(cudaStreamSynchronize(st));
  GR_CK(cudaGetLastError());
  return LRB_OK;
}

}  // namespace lrb

namespace lrb {

// cuBLAS handle of the current device, created on first use and kept until
// exit.
cublasHandle_t grad_blas() {
  static std::mutex mu;
  static std::vector<cublasHandle_t> h;   // indexed by device
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if ((size_t)dev >= h.size()) h.resize((size_t)dev + 1, nullptr);
  if (!h[dev]) cublasCreate(&h[dev]);
  return h[dev];
}

}  // namespace lrb
