// One-electron integrals S, T, V on the GPU (needed to keep the SCF on the
// device; O(n^2) work).  Same operators and normalisation as the reference's
// cint1e_ovlp/kin/nuc (src/cint1e.rs:925,976; src/intor1.rs:168;
// src/g1e.rs:241-330): overlap by the Obara-Saika 1D recurrence, kinetic as
// -1/2 d^2/dx^2 on the ket, nuclear attraction by Rys quadrature with
// (li+lj)/2+1 roots per point nucleus.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include <cuda_runtime.h>

#include "engine.h"
#include "eri_device.cuh"

namespace lrb {

const double *rys_table_device();

namespace {

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

// 1D overlap s(i, j) for i <= imax, j <= jmax (s(0,0) = 1); returns s(ti, tj).
__device__ double os_1d(int ti, int tj, double xpa, double xpb, double oo2p) {
  double s[5][7];   // i <= 4, j <= 6 (kinetic needs j + 2)
  for (int i = 0; i <= ti; ++i)
    for (int j = 0; j <= tj; ++j) {
      double v;
      if (i == 0 && j == 0) {
        v = 1.0;
      } else if (i > 0) {
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

template <int NR>
__device__ void nuc_roots(const double *tab, double x, double *u, double *w) {
  for (int f = 0; f < 2 * NR; ++f) {
    const double v = rys_function<NR>(tab, x, f);
    if (f < NR) u[f] = v; else w[f - NR] = v;
  }
}

// One thread per cartesian AO pair (mu, nu): typec 0 S, 1 T, 2 V.
__global__ void k_int1e_cart(int typec, int n, const int *__restrict__ ao_shell,
                             const int *__restrict__ ao_comp, const int *__restrict__ atm,
                             int natm, const int *__restrict__ bas,
                             const double *__restrict__ env, const double *__restrict__ rys,
                             double *out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int mu = (int)(t / n), nu = (int)(t % n);
  const int si = ao_shell[mu], sj = ao_shell[nu];
  const int *bi = bas + 8 * si, *bj = bas + 8 * sj;
  const int li = bi[1], lj = bj[1];
  int ia[3], jb[3];
  cart_of(li, ao_comp[mu], ia[0], ia[1], ia[2]);
  cart_of(lj, ao_comp[nu], jb[0], jb[1], jb[2]);
  const double *A = env + atm[6 * bi[0] + 1], *Bc = env + atm[6 * bj[0] + 1];
  const double rab2 = (A[0] - Bc[0]) * (A[0] - Bc[0]) + (A[1] - Bc[1]) * (A[1] - Bc[1]) +
                      (A[2] - Bc[2]) * (A[2] - Bc[2]);
  const double cfac = fac_sp(li) * fac_sp(lj);
  double acc = 0.0;
  for (int jp = 0; jp < bj[2]; ++jp)
    for (int ip = 0; ip < bi[2]; ++ip) {
      const double ai = env[bi[5] + ip], bjx = env[bj[5] + jp], p = ai + bjx;
      const double mu_ = ai * bjx / p;
      const double cc = env[bi[6] + ip] * env[bj[6] + jp] * cfac * exp(-mu_ * rab2);
      double P[3];
      for (int d = 0; d < 3; ++d) P[d] = (ai * A[d] + bjx * Bc[d]) / p;
      if (typec == 0 || typec == 1) {
        const double pre = cc * pow(M_PI / p, 1.5);
        double s1[3];
        for (int d = 0; d < 3; ++d) s1[d] = os_1d(ia[d], jb[d], P[d] - A[d], P[d] - Bc[d], 0.5 / p);
        if (typec == 0) {
          acc += pre * s1[0] * s1[1] * s1[2];
        } else {
          double v = 0.0;
          for (int d = 0; d < 3; ++d) {
            const int j = jb[d];
            double tt = -2.0 * bjx * (2 * j + 1) * s1[d] +
                        4.0 * bjx * bjx * os_1d(ia[d], j + 2, P[d] - A[d], P[d] - Bc[d], 0.5 / p);
            if (j >= 2) tt += j * (j - 1) * os_1d(ia[d], j - 2, P[d] - A[d], P[d] - Bc[d], 0.5 / p);
            tt *= -0.5;
            double o = 1.0;
            for (int e = 0; e < 3; ++e)
              if (e != d) o *= s1[e];
            v += tt * o;
          }
          acc += pre * v;
        }
      } else {
        const int lsum = li + lj, nr = lsum / 2 + 1;
        for (int c = 0; c < natm; ++c) {
          const double *C = env + atm[6 * c + 1];
          const double z = -fabs((double)atm[6 * c]);
          const double pc2 = (P[0] - C[0]) * (P[0] - C[0]) + (P[1] - C[1]) * (P[1] - C[1]) +
                             (P[2] - C[2]) * (P[2] - C[2]);
          double u[5], w[5];
          const double x = p * pc2;
          switch (nr) {
            case 1: nuc_roots<1>(rys + rys_tab_offset(1), x, u, w); break;
            case 2: nuc_roots<2>(rys + rys_tab_offset(2), x, u, w); break;
            case 3: nuc_roots<3>(rys + rys_tab_offset(3), x, u, w); break;
            case 4: nuc_roots<4>(rys + rys_tab_offset(4), x, u, w); break;
            default: nuc_roots<5>(rys + rys_tab_offset(5), x, u, w); break;
          }
          const double pre = cc * 2.0 * M_PI / p * z;
          for (int r = 0; r < nr; ++r) {
            const double t2 = u[r] / (1.0 + u[r]);
            double prod = 1.0;
            for (int d = 0; d < 3; ++d) {
              // I(n+1) = (PA - t2 PC) I(n) + n/(2p)(1 - t2) I(n-1); then
              // I(i, j) = sum_k C(j,k) (A-B)^(j-k) I(i+k)
              double g[9];
              g[0] = 1.0;
              const double c0 = (P[d] - A[d]) - t2 * (P[d] - C[d]);
              const double b1 = 0.5 / p * (1.0 - t2);
              const int top = ia[d] + jb[d];
              if (top > 0) g[1] = c0;
              for (int k = 1; k < top; ++k) g[k + 1] = c0 * g[k] + k * b1 * g[k - 1];
              const double ab = A[d] - Bc[d];
              double v = 0.0, binc = 1.0, pw = 1.0;
              // sum over k = j..0 of C(j,k) ab^(j-k) g[i+k]
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
      }
    }
  out[t] = acc;
}

// Cartesian -> spherical for a matrix: out[mu_s][nu_s] = sum c2s c2s M_cart.
__constant__ double c_c2s1[5 * 9 * 15];
__global__ void k_mat_cart2sph(int ns, int nc, const int *__restrict__ sph_shell,
                               const int *__restrict__ sph_m, const int *__restrict__ cart_off,
                               const int *__restrict__ bas, const double *__restrict__ M,
                               double *out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ns * ns) return;
  const int a = (int)(t / ns), b = (int)(t % ns);
  const int si = sph_shell[a], sj = sph_shell[b];
  const int li = bas[8 * si + 1], lj = bas[8 * sj + 1];
  const int ma = sph_m[a], mb = sph_m[b];
  double v = 0.0;
  for (int ca = 0; ca < ncart(li); ++ca) {
    const double x = c_c2s1[(li * 9 + ma) * 15 + ca];
    if (x == 0.0) continue;
    for (int cb = 0; cb < ncart(lj); ++cb) {
      const double y = c_c2s1[(lj * 9 + mb) * 15 + cb];
      if (y == 0.0) continue;
      v += x * y * M[(long long)(cart_off[a] + ca) * nc + cart_off[b] + cb];
    }
  }
  out[t] = v;
}

}  // namespace

// n x n one-electron matrix on the device (coord 0 cartesian, 1 spherical).
// d_* are device copies of the molecule; out is a device buffer of n*n.
int int1e_device(int typec, int coord, const int *d_atm, int natm, const int *d_bas, int nbas,
                 const double *d_env, const int *h_bas, double *out, cudaStream_t st,
                 const double *c2s_host) {
  // AO maps on the host (small)
  std::vector<int> ao_shell, ao_comp, sph_shell, sph_m, cart_off_of_sph;
  std::vector<int> cart_start(nbas);
  for (int s = 0; s < nbas; ++s) {
    const int l = h_bas[8 * s + 1];
    if (h_bas[8 * s + 3] != 1 || l > 4) return set_error("int1e: nctr != 1 or l > 4"), LRB_ERR_UNSUPPORTED;
    cart_start[s] = (int)ao_shell.size();
    for (int c = 0; c < ncart(l); ++c) { ao_shell.push_back(s); ao_comp.push_back(c); }
    for (int m = 0; m < nsph(l); ++m) {
      sph_shell.push_back(s); sph_m.push_back(m); cart_off_of_sph.push_back(cart_start[s]);
    }
  }
  const int nc = (int)ao_shell.size(), ns = (int)sph_shell.size();
  int *buf = nullptr;
  const size_t ni = 2 * (size_t)nc + 3 * (size_t)ns;
  double *mc = nullptr;
  if (cudaMallocAsync((void **)&buf, sizeof(int) * ni, st) != cudaSuccess)
    return set_error("int1e: allocation failed"), LRB_ERR_ALLOC;
  int *d_shell = buf, *d_comp = buf + nc, *d_sshell = buf + 2 * nc, *d_sm = d_sshell + ns,
      *d_coff = d_sm + ns;
  cudaMemcpyAsync(d_shell, ao_shell.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_comp, ao_comp.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_sshell, sph_shell.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_sm, sph_m.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_coff, cart_off_of_sph.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st);
  double *target = out;
  if (coord == 1) {
    if (cudaMallocAsync((void **)&mc, sizeof(double) * (size_t)nc * nc, st) != cudaSuccess) {
      cudaFreeAsync(buf, st);
      return set_error("int1e: allocation failed"), LRB_ERR_ALLOC;
    }
    target = mc;
  }
  const long long tot = (long long)nc * nc;
  k_int1e_cart<<<(unsigned)((tot + 127) / 128), 128, 0, st>>>(
      typec, nc, d_shell, d_comp, d_atm, natm, d_bas, d_env, rys_table_device(), target);
  engine().launches++;
  if (coord == 1) {
    cudaMemcpyToSymbolAsync(c_c2s1, c2s_host, sizeof(c_c2s1), 0, cudaMemcpyHostToDevice, st);
    const long long ts = (long long)ns * ns;
    k_mat_cart2sph<<<(unsigned)((ts + 127) / 128), 128, 0, st>>>(ns, nc, d_sshell, d_sm, d_coff,
                                                                 d_bas, mc, out);
    engine().launches++;
    cudaFreeAsync(mc, st);
  }
  cudaFreeAsync(buf, st);
  if (cudaGetLastError() != cudaSuccess) return set_error("int1e: launch failed"), LRB_ERR_CUDA;
  return LRB_OK;
}

}  // namespace lrb
