// RHF SCF on the GPU (cartesian AOs, like the reference's src/scf.rs).
//
// Reference algorithm (src/scf.rs:743-799): X = U s^-1/2 from the overlap
// (refuse s_min < 1e-8), P0 = I, plain Roothaan iteration F = H + G(P),
// F' = X^T F X, eigh (ascending), C = X U, P = 2 C_occ C_occ^T, until
// ||P - P_old||_F / 2 <= conv; then the density checks tr(PS) = N and
// PSP = 2P (1e-6) and E = sum P (H + F) / 2 + E_nn (src/scf.rs:801-956).
// Options add the core-Hamiltonian guess, a caller-supplied P0 and DIIS
// (FP64, error FPS - SPF), none of which changes the converged energy.
// Dense algebra: cuBLAS dgemm and cuSOLVER dsyevd; matrices column-major
// (all symmetric ones are layout-free).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "fock.h"

namespace lrb {

void fill_c2s(double *c);

namespace {

struct Handles {
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
};

// cuBLAS / cuSOLVER handles of the current device, created on first use and
// kept until exit.
Handles &handles() {
  static std::mutex mu;
  static std::vector<Handles *> h;   // indexed by device
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if ((size_t)dev >= h.size()) h.resize((size_t)dev + 1, nullptr);
  if (!h[dev]) {
    h[dev] = new Handles();
    cublasCreate(&h[dev]->blas);
    cusolverDnCreate(&h[dev]->sol);
  }
  return *h[dev];
}

__global__ void k_axpby(const double *a, const double *b, double *c, double alpha, double beta,
                        long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) c[t] = alpha * a[t] + beta * b[t];
}

__global__ void k_scale_cols(double *U, const double *s, int n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int col = (int)(t / n);
  U[t] *= 1.0 / sqrt(s[col]);
}

__global__ void k_identity(double *P, int n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  P[t] = (t / n == t % n) ? 1.0 : 0.0;
}

// block-wide sum of x[i]*y[i] (two-stage through atomics, FP64)
__global__ void k_dot(const double *x, const double *y, long long n, double *out) {
  __shared__ double sm[256];
  double s = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    s += x[t] * y[t];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, sm[0]);
}

__global__ void k_absmax_diff2(const double *a, const double *b, long long n, double *out) {
  // out = max |a - 2 b|
  __shared__ double sm[256];
  double s = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    s = fmax(s, fabs(a[t] - 2.0 * b[t]));
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(sm[0]));
  }
}

struct Dev {
  cudaStream_t st;
  std::vector<void *> owned;
  bool ok = true;
  template <class T>
  T *alloc(size_t n) {
    void *p = nullptr;
    if (cudaMallocAsync(&p, std::max(n, (size_t)1) * sizeof(T), st) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    owned.push_back(p);
    return (T *)p;
  }
  ~Dev() {
    for (void *p : owned) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
  }
};

// eigh in place: A (n x n, symmetric) -> eigenvectors (columns), w ascending
int eigh(int n, double *A, double *w, cudaStream_t st, Dev &dv) {
  Handles &h = handles();
  cusolverDnSetStream(h.sol, st);
  int lwork = 0;
  if (cusolverDnDsyevd_bufferSize(h.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n,
                                  w, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return set_error("cusolver bufferSize failed"), LRB_ERR_CUDA;
  double *work = dv.alloc<double>(lwork);
  int *info = dv.alloc<int>(1);
  if (!dv.ok) return set_error("scf: allocation failed"), LRB_ERR_ALLOC;
  if (cusolverDnDsyevd(h.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n, w, work,
                       lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return set_error("cusolver dsyevd failed"), LRB_ERR_CUDA;
  int hinfo = 0;
  cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (hinfo != 0) return set_error("eigensolver did not converge"), LRB_ERR_SCF;
  return LRB_OK;
}

// C = op(A) * op(B), column-major
void gemm(cublasOperation_t ta, cublasOperation_t tb, int m, int nn, int k, const double *A,
          int lda, const double *B, int ldb, double *C, int ldc, double beta = 0.0,
          double alpha = 1.0) {
  cublasDgemm(handles().blas, ta, tb, m, nn, k, &alpha, A, lda, B, ldb, &beta, C, ldc);
}

double dot(const double *x, const double *y, long long n, cudaStream_t st, double *scratch) {
  cudaMemsetAsync(scratch, 0, sizeof(double), st);
  k_dot<<<256, 256, 0, st>>>(x, y, n, scratch);
  double h = 0.0;
  cudaMemcpyAsync(&h, scratch, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return h;
}

double nuclear_repulsion(const MolCtx &m) {
  double e = 0.0;
  for (int i = 0; i < m.natm; ++i)
    for (int j = 0; j < i; ++j) {
      const double *ri = &m.h_env[m.h_atm[6 * i + 1]], *rj = &m.h_env[m.h_atm[6 * j + 1]];
      const double d = std::sqrt((ri[0] - rj[0]) * (ri[0] - rj[0]) + (ri[1] - rj[1]) * (ri[1] - rj[1]) +
                                 (ri[2] - rj[2]) * (ri[2] - rj[2]));
      e += (double)(m.h_atm[6 * i] * m.h_atm[6 * j]) / d;
    }
  return e;
}

// Small dense solve (DIIS normal equations, <= 9 unknowns) by Gaussian
// elimination with partial pivoting.
bool solve_small(int n, std::vector<double> A, std::vector<double> &b) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (std::fabs(A[p * n + c]) < 1e-300) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[p * n + k]);
      std::swap(b[c], b[p]);
    }
    for (int r = c + 1; r < n; ++r) {
      const double f = A[r * n + c] / A[c * n + c];
      for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double s = b[c];
    for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
    b[c] = s / A[c * n + c];
  }
  return true;
}

}  // namespace

int scf_run(MolCtx &m, size_t nelec, const ScfOptions &o, ScfResult *res, double *h_P_out,
            const double *h_P0, cudaStream_t st) {
  const auto t0 = std::chrono::steady_clock::now();
  const int n = m.nao;
  const long long nn = (long long)n * n;
  const int nocc = (int)(nelec / 2);
  if (nelec % 2 || nocc > n || nocc < 1) return set_error("scf: need an even electron count <= 2 nao"), LRB_ERR_INPUT;
  Dev dv{st};
  double *S = dv.alloc<double>(nn), *T = dv.alloc<double>(nn), *V = dv.alloc<double>(nn);
  double *H = dv.alloc<double>(nn), *X = dv.alloc<double>(nn), *P = dv.alloc<double>(nn);
  double *Pold = dv.alloc<double>(nn), *G = dv.alloc<double>(nn), *F = dv.alloc<double>(nn);
  double *W1 = dv.alloc<double>(nn), *W2 = dv.alloc<double>(nn), *C = dv.alloc<double>(nn);
  double *ev = dv.alloc<double>(n), *scr = dv.alloc<double>(2);
  const int ndiis = o.diis > 0 ? std::min(o.diis, 20) : 0;
  double *Fh = ndiis ? dv.alloc<double>(nn * ndiis) : nullptr;
  double *Eh = ndiis ? dv.alloc<double>(nn * ndiis) : nullptr;
  if (!dv.ok) return set_error("scf: device allocation failed"), LRB_ERR_ALLOC;
  Handles &h = handles();
  cublasSetStream(h.blas, st);
  double c2s[5 * 9 * 15];
  fill_c2s(c2s);
  int rc = int1e_device(0, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), S, st, c2s);
  if (!rc) rc = int1e_device(1, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), T, st, c2s);
  if (!rc) rc = int1e_device(2, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), V, st, c2s);
  if (rc) return rc;
  const unsigned gb = (unsigned)((nn + 255) / 256);
  k_axpby<<<gb, 256, 0, st>>>(T, V, H, 1.0, 1.0, nn);
  // X = U s^-1/2
  cudaMemcpyAsync(X, S, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
  if ((rc = eigh(n, X, ev, st, dv))) return rc;
  double smin = 0.0;
  cudaMemcpyAsync(&smin, ev, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (smin < 1e-8) return set_error("overlap matrix is near-singular (smallest eigenvalue < 1e-8)"), LRB_ERR_SCF;
  k_scale_cols<<<gb, 256, 0, st>>>(X, ev, n);

  auto density_from_fock = [&](const double *Fm) -> int {
    // F' = X^T F X ; eigh ; C = X U ; P = 2 C_occ C_occ^T
    gemm(CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, X, n, Fm, n, W1, n);
    gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, W1, n, X, n, W2, n);
    int r = eigh(n, W2, ev, st, dv);
    if (r) return r;
    gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, X, n, W2, n, C, n);
    gemm(CUBLAS_OP_N, CUBLAS_OP_T, n, n, nocc, C, n, C, n, P, n, 0.0, 2.0);
    return LRB_OK;
  };

  // initial density
  if (h_P0) {
    cudaMemcpyAsync(P, h_P0, sizeof(double) * nn, cudaMemcpyHostToDevice, st);
  } else if (o.guess == 1) {
    if ((rc = density_from_fock(H))) return rc;
  } else {
    k_identity<<<gb, 256, 0, st>>>(P, n);   // reference P0 = I (src/scf.rs:757-764)
  }
  double delta = 1.0;
  int it = 0;
  int nd = 0;
  double fock_ms = 0.0;
  long long quartets = 0, q32 = 0;
  // incremental (mixed) mode: Gc holds G(Pb), Pb the density it was built for
  double *Gc = o.mixed ? dv.alloc<double>(nn) : nullptr;
  double *Pb = o.mixed ? dv.alloc<double>(nn) : nullptr;
  double *dPm = o.mixed ? dv.alloc<double>(nn) : nullptr;
  if (!dv.ok) return set_error("scf: device allocation failed"), LRB_ERR_ALLOC;
  // mixed schedule: phase 1 all FP32 while the density moves by more than
  // fp32_until (left for good when it stops shrinking below 10 x
  // fp32_until), phase 2 FP32 only
  // for quartets with bound < tau32, phase 0 all FP64 once ||dP||/2 is within
  // 10 x conv, so the last iterations and the fixed point are those of the
  // FP64 operator.  A phase change forces a full build; leaving phase 1
  // restarts DIIS.
  int since_full = 1 << 30, phase = -1;
  bool fp32_done = false, fp64_final = false;
  double hist[3] = {1e300, 1e300, 1e300};   // delta of the last iterations
  // LRB_SCF_TRACE=1: one line per iteration on stderr (phase, build kind,
  // quartets, build time, DIIS depth, density change)
  static const bool trace = getenv("LRB_SCF_TRACE") && atoi(getenv("LRB_SCF_TRACE")) > 0;
  while (delta > o.conv && it < o.max_iter) {
    cudaMemcpyAsync(Pold, P, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
    const auto tf = std::chrono::steady_clock::now();
    FockStats fs;
    if (!o.mixed) {
      if ((rc = fock_build(m, P, G, o.tau, st, &fs))) return rc;
    } else {
      // no progress in two steps: the FP32 operator's error floor, which
      // lies near fp32_until; far above it a stall is the iteration's own
      // (DIIS between two basins) and FP64 builds would not end it sooner
      if (it >= 3 && delta > 0.5 * hist[2] && delta < 10.0 * o.fp32_until) fp32_done = true;
      if (it > 0 && delta <= o.fp32_until) fp32_done = true;
      if (fp32_done && delta <= 10.0 * o.conv) fp64_final = true;
      const int want = !fp32_done ? 1 : (fp64_final ? 0 : 2);
      const bool full = want != phase || since_full >= o.rebuild_every;
      // DIIS restarts when the all-FP32 phase ends: its Fock matrices carry
      // the FP32 error.  The split phase differs from FP64 only in quartets
      // below tau32, so its history stays valid for the FP64 phase.
      if (want != phase && phase == 1) nd = 0;
      // the FP32 phases screen at tau_fp32: their G carries the FP32 error
      // already, and the FP64 phase starts with a full build at tau
      const double tau_b = want == 0 ? o.tau : std::max(o.tau, o.tau_fp32);
      if (full) {
        if ((rc = fock_build(m, P, Gc, tau_b, st, &fs, want, o.tau32, false))) return rc;
        since_full = 0;
        phase = want;
      } else {
        k_axpby<<<gb, 256, 0, st>>>(P, Pb, dPm, 1.0, -1.0, nn);
        if ((rc = fock_build(m, dPm, Gc, tau_b, st, &fs, phase, o.tau32, true))) return rc;
        ++since_full;
      }
      cudaMemcpyAsync(Pb, P, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(G, Gc, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
    }
    quartets += fs.quartets;
    q32 += fs.fp32_quartets;
    k_axpby<<<gb, 256, 0, st>>>(H, G, F, 1.0, 1.0, nn);
    cudaStreamSynchronize(st);
    fock_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf).count();
    const double build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf).count();
    const double *Fuse = F;
    if (ndiis) {
      // error e = F P S - S P F, stored in slot it % ndiis
      const int slot = nd % ndiis;
      double *e = Eh + nn * slot;
      gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, F, n, P, n, W1, n);
      gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, W1, n, S, n, e, n);
      gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, S, n, P, n, W1, n);
      gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, W1, n, F, n, e, n, 1.0, -1.0);
      cudaMemcpyAsync(Fh + nn * slot, F, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
      ++nd;
      const int k = std::min(nd, ndiis);
      if (k >= 2) {
        std::vector<double> A((k + 1) * (k + 1), 0.0), b(k + 1, 0.0);
        for (int i = 0; i < k; ++i)
          for (int j = 0; j <= i; ++j) {
            const double v = dot(Eh + nn * i, Eh + nn * j, nn, st, scr);
            A[i * (k + 1) + j] = A[j * (k + 1) + i] = v;
          }
        for (int i = 0; i < k; ++i) A[i * (k + 1) + k] = A[k * (k + 1) + i] = -1.0;
        b[k] = -1.0;
        if (solve_small(k + 1, A, b)) {
          cudaMemsetAsync(W1, 0, sizeof(double) * nn, st);
          for (int i = 0; i < k; ++i)
            k_axpby<<<gb, 256, 0, st>>>(W1, Fh + nn * i, W1, 1.0, b[i], nn);
          Fuse = W1;
          cudaMemcpyAsync(G, W1, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
          Fuse = G;
        }
      }
    }
    if ((rc = density_from_fock(Fuse))) return rc;
    k_axpby<<<gb, 256, 0, st>>>(P, Pold, W1, 1.0, -1.0, nn);
    delta = std::sqrt(dot(W1, W1, nn, st, scr)) / 2.0;
    if (trace)
      fprintf(stderr, "scf it %3d phase %2d %s quartets %11lld fp32 %11lld build %8.1f ms diis %d delta %.3e\n",
              it, o.mixed ? phase : 0, o.mixed && since_full > 0 ? "incr" : "full", fs.quartets,
              fs.fp32_quartets, build_ms, ndiis ? std::min(nd, ndiis) : 0, delta);
    hist[2] = hist[1];
    hist[1] = hist[0];
    hist[0] = delta;
    ++it;
  }
  if (res) {
    res->iterations = it;
    res->delta = delta;
    res->converged = delta <= o.conv;
    res->quartets = quartets;
    res->fp32_quartets = q32;
    res->fock_ms = fock_ms;
  }
  if (delta > o.conv) return set_error("SCF did not converge"), LRB_ERR_SCF;
  // density checks (src/scf.rs:572-600)
  const double tr = dot(P, S, nn, st, scr);   // tr(PS) for symmetric P, S
  gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, P, n, S, n, W1, n);
  gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, W1, n, P, n, W2, n);
  cudaMemsetAsync(scr, 0, sizeof(double), st);
  k_absmax_diff2<<<256, 256, 0, st>>>(W2, P, nn, scr);
  double idem = 0.0;
  cudaMemcpyAsync(&idem, scr, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (std::fabs(tr - (double)nelec) > 1e-6 || idem > 1e-6)
    return set_error("converged density failed tr(PS) = N or PSP = 2P"), LRB_ERR_SCF;
  // energy at the final density: sum P (H + F)/2 + E_nn with F = H + G(P)
  FockStats fs;
  if ((rc = fock_build(m, P, G, o.tau, st, &fs))) return rc;
  const double e1 = dot(P, H, nn, st, scr);
  const double e2 = dot(P, G, nn, st, scr);
  const double enuc = nuclear_repulsion(m);
  if (res) {
    res->energy = e1 + 0.5 * e2 + enuc;
    res->e_nuc = enuc;
    res->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (h_P_out) {
    cudaMemcpyAsync(h_P_out, P, sizeof(double) * nn, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
  }
  return LRB_OK;
}

// Energy functional at a given density (reference energyfast, src/scf.rs:827).
int energy_at(MolCtx &m, const double *h_P, double tau, double *E, cudaStream_t st) {
  const int n = m.nao;
  const long long nn = (long long)n * n;
  Dev dv{st};
  double *T = dv.alloc<double>(nn), *V = dv.alloc<double>(nn), *P = dv.alloc<double>(nn);
  double *G = dv.alloc<double>(nn), *scr = dv.alloc<double>(2);
  if (!dv.ok) return set_error("energy: allocation failed"), LRB_ERR_ALLOC;
  double c2s[5 * 9 * 15];
  fill_c2s(c2s);
  int rc = int1e_device(1, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), T, st, c2s);
  if (!rc) rc = int1e_device(2, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), V, st, c2s);
  if (rc) return rc;
  cudaMemcpyAsync(P, h_P, sizeof(double) * nn, cudaMemcpyHostToDevice, st);
  if ((rc = fock_build(m, P, G, tau, st, nullptr))) return rc;
  const double et = dot(P, T, nn, st, scr), ev = dot(P, V, nn, st, scr), eg = dot(P, G, nn, st, scr);
  *E = et + ev + 0.5 * eg + nuclear_repulsion(m);
  return LRB_OK;
}

}  // namespace lrb

namespace lrb {

// F = T + V + G(P) with every quartet in FP64 (no screening).
int scf_dense_fock(MolCtx &m, const double *P, double *F, cudaStream_t st) {
  const long long nn = (long long)m.nao * m.nao;
  double *T = nullptr, *V = nullptr, *G = nullptr;
  if (cudaMallocAsync((void **)&T, sizeof(double) * nn, st) != cudaSuccess ||
      cudaMallocAsync((void **)&V, sizeof(double) * nn, st) != cudaSuccess ||
      cudaMallocAsync((void **)&G, sizeof(double) * nn, st) != cudaSuccess)
    return set_error("fock: allocation failed"), LRB_ERR_ALLOC;
  double c2s[5 * 9 * 15];
  fill_c2s(c2s);
  int rc = int1e_device(1, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), T, st, c2s);
  if (!rc) rc = int1e_device(2, 0, m.atm, m.natm, m.bas, m.nbas, m.env, m.h_bas.data(), V, st, c2s);
  if (!rc) rc = fock_build(m, P, G, 0.0, st, nullptr);
  if (!rc) {
    const unsigned gb = (unsigned)((nn + 255) / 256);
    k_axpby<<<gb, 256, 0, st>>>(T, V, F, 1.0, 1.0, nn);
    k_axpby<<<gb, 256, 0, st>>>(F, G, F, 1.0, 1.0, nn);
  }
  cudaFreeAsync(T, st);
  cudaFreeAsync(V, st);
  cudaFreeAsync(G, st);
  return rc;
}

}  // namespace lrb
