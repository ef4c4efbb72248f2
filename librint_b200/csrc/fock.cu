// Direct Fock build G(P) on the GPU: the reference's integral2e_fock
// (src/scf.rs:316-410) without the dense tensor and with 8-fold symmetry.
//
//  * molecule context: device copies of atm/bas/env, AO offsets, and a pair
//    table of all shell pairs I >= J (oriented l_first >= l_second) with their
//    primitive pairs and Schwarz factors Q_IJ = sqrt(max |(ab|ab)|);
//  * per build: shell-block density maxima, quartet screening
//    Q_IJ Q_KL max(2D_IJ, 2D_KL, D_IK, D_IL, D_JK, D_JL) >= tau over canonical
//    pair pairs, compaction into a job list sorted by class and primitive
//    count, per-class digestion kernels (k_eri<..., 1>), symmetrisation.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <vector>

#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "eri_classes.cuh"
#include "fock.h"

namespace lrb {

const double *rys_table_device();

#define FK_CK(x)                                  \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) {                      \
      set_error(cudaGetErrorString(e_));          \
      return LRB_ERR_CUDA;                        \
    }                                             \
  } while (0)

namespace {

// Quartets with at least this many primitive quartets run one lane per
// primitive quartet where the class has that kernel (LRB_FOCK_LP_MIN or
// lrb_fock_lane_min override it; 0x100000 turns the lane kernels off).
std::atomic<int> g_lp_min{0};
int fock_lp_min() {
  int v = g_lp_min.load();
  if (v == 0) {
    const char *e = getenv("LRB_FOCK_LP_MIN");
    const long x = e ? strtol(e, nullptr, 10) : LP_MIN_PRIM;
    v = (int)std::min(std::max(x, 1L), 0x100000L);
    int z = 0;
    if (!g_lp_min.compare_exchange_strong(z, v)) v = z;
  }
  return v;
}

__device__ inline double fac_sp_d(int l) {
  return l == 0 ? 0.28209479177387814 : (l == 1 ? 0.48860251190291992 : 1.0);
}

// Primitive pairs of every table pair (one thread per primitive pair).
// sqrt(2 pi^2.5) is folded into every pair so bra.fac * ket.fac carries the
// class prefactor 2 pi^3 / sqrt(pi) (reference src/g2e.rs:74-82).
__global__ void k_mol_pairs(const PairInfo *__restrict__ pairs, int npairs,
                            const int *__restrict__ atm, const int *__restrict__ bas,
                            const double *__restrict__ env, PrimPair *pp, int npp_total,
                            int gc_screen) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npp_total) return;
  int lo = 0, hi = npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pairs[mid].pp_off <= t) lo = mid; else hi = mid - 1;
  }
  const PairInfo pr = pairs[lo];
  const int *bi = bas + 8 * pr.ish, *bj = bas + 8 * pr.jsh;
  const int ki = bi[2], kj = bj[2];
  const int e = t - pr.pp_off;
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
  o.fac = ci * cj * exp(-eij) * fac_sp_d(bi[1]) * fac_sp_d(bj[1]) * 5.9149671727956129;
  o.ia = 1.0 / aij;
  o.facia = o.fac * o.ia;
  // sub-shells of generally contracted shells screen with the largest
  // |coefficient| over the contractions (bas slot 7)
  const double sci = gc_screen && bi[7] > 0 ? env[bi[7] + ip] : ci;
  const double scj = gc_screen && bj[7] > 0 ? env[bj[7] + jp] : cj;
  o.cce = eij - log_rr - log(fabs(sci)) - log(fabs(scj));
  pp[t] = o;
}

// Q_IJ from the diagonal of the (IJ|IJ) cartesian blocks.
__global__ void k_schwarz(const double *__restrict__ blocks, const long long *__restrict__ boff,
                          const int *__restrict__ dims, int npairs, double *Q) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int ni = dims[2 * p], nj = dims[2 * p + 1];
  const double *b = blocks + boff[p];
  double m = 0.0;
  for (int a = 0; a < ni; ++a)
    for (int c = 0; c < nj; ++c) {
      const long long e = a + (long long)ni * (c + (long long)nj * (a + (long long)ni * c));
      m = fmax(m, fabs(b[e]));
    }
  Q[p] = sqrt(m);
}

// log of each primitive pair's Schwarz factor, sqrt(max |(ab|ab)|) over the
// cartesian components of its (ij|ij) block (float; -inf when zero).
__global__ void k_prim_schwarz(const double *__restrict__ blocks, const long long *__restrict__ roff,
                               const int *__restrict__ rdim, int nrec, float *lq) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  const int ni = rdim[2 * r], nj = rdim[2 * r + 1];
  const double *b = blocks + roff[r];
  double m = 0.0;
  for (int a = 0; a < ni; ++a)
    for (int c = 0; c < nj; ++c) {
      const long long e = a + (long long)ni * (c + (long long)nj * (a + (long long)ni * c));
      m = fmax(m, fabs(b[e]));
    }
  lq[r] = m > 0.0 ? (float)(0.5 * log(m)) : -INFINITY;
}

// Shell-block maxima of |P|.
__global__ void k_dens_max(const double *__restrict__ P, int n, const int *__restrict__ aooff,
                           int nbas, double *Dsh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbas * nbas) return;
  const int I = t / nbas, J = t % nbas;
  double m = 0.0;
  for (int a = aooff[I]; a < aooff[I + 1]; ++a)
    for (int b = aooff[J]; b < aooff[J + 1]; ++b) m = fmax(m, fabs(P[(long long)a * n + b]));
  Dsh[t] = m;
}

// Largest shell-block density maximum (one block).
__global__ void k_max_reduce(const double *__restrict__ v, int n, double *out) {
  __shared__ double sm[1024];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, v[i]);
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sm[0];
}

// Candidate count per sorted bra position i: ket positions j <= i whose
// Q_i Q_j 2 Dmax reaches tau (a prefix, as Qs is descending).  2 Dmax bounds
// the density factor of every quartet, so nothing the full test keeps is lost.
__global__ void k_cand_count(const double *__restrict__ Qs, int npairs,
                             const double *__restrict__ dmax, double tau, int *cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  const double f = Qs[i] * 2.0 * dmax[0];
  int c = 0;
  if (f > 0.0) {
    const double thr = tau / f;
    int lo = 0, hi = i + 1;   // first j in [0, i] with Qs[j] < thr
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (Qs[mid] >= thr) lo = mid + 1; else hi = mid;
    }
    c = lo;
  }
  cnt[i] = c;
}

// Screen the candidates (sorted positions i >= j) and append survivors: a
// quartet is kept when Q_IJ Q_KL max(2|D_IJ|, 2|D_KL|, |D_IK|, |D_IL|,
// |D_JK|, |D_JL|) >= tau, runs in FP32 for prec 1 (or prec 2 with the bound
// below tau32), and is keyed by (precision, class, primitive count) for the
// radix sort that groups the class launches.
__global__ void k_screen_sorted(const PairInfo *__restrict__ pairs, const int *__restrict__ pcls,
                                const double *__restrict__ Q, const int *__restrict__ qorder,
                                const long long *__restrict__ qoff, int npairs,
                                const double *__restrict__ Dsh, int nbas, long long ncand,
                                double tau, int prec, double tau32, int rank, int nranks,
                                int2 *jobs, unsigned *keys, int *idx, unsigned long long *count,
                                unsigned long long cap) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  bool keep = false;
  int b = 0, k = 0;
  unsigned key = 0;
  // a rank takes the candidates t = rank (mod nranks): the candidate index is
  // a function of the Schwarz-sorted pair positions only, so every rank
  // enumerates the same list and the shares are disjoint and complete
  if (t < ncand && t % nranks == rank) {
    int lo = 0, hi = npairs - 1;   // last position i with qoff[i] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (qoff[mid] <= t) lo = mid; else hi = mid - 1;
    }
    b = qorder[lo];
    k = qorder[(int)(t - qoff[lo])];
    const PairInfo pb = pairs[b], pk = pairs[k];
    const int I = pb.ish, J = pb.jsh, K = pk.ish, L = pk.jsh;
    const double d = fmax(fmax(2.0 * Dsh[I * nbas + J], 2.0 * Dsh[K * nbas + L]),
                          fmax(fmax(Dsh[I * nbas + K], Dsh[I * nbas + L]),
                               fmax(Dsh[J * nbas + K], Dsh[J * nbas + L])));
    const double bound = Q[b] * Q[k] * d;
    keep = bound >= tau;
    if (keep) {
      int cb = pcls[b], ck = pcls[k];
      if (cb < ck) {
        const int tmp = b; b = k; k = tmp;
        const int tc = cb; cb = ck; ck = tc;
      }
      const int cid0 = cb * (cb + 1) / 2 + ck;
      // classes with an f shell have FP64 kernels only
      const bool f32 = (prec == 1 || (prec == 2 && bound < tau32)) && cid0 < NCLASS_TPL;
      const int cid = cid0 + (f32 ? NCLASS : 0);
      const int kprod = pairs[b].npp * pairs[k].npp;
      key = ((unsigned)cid << 20) | (unsigned)(0xfffff - kprod);
    }
  }
  const unsigned mask = __ballot_sync(0xffffffffu, keep);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  unsigned long long base = 0;
  if (lane == __ffs(mask) - 1) base = atomicAdd(count, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
  if (keep) {
    const unsigned long long pos = base + __popc(mask & ((1u << lane) - 1));
    if (pos < cap) {
      jobs[pos] = make_int2(b, k);
      keys[pos] = key;
      idx[pos] = (int)pos;
    }
  }
}

// starts[c] = first sorted position whose key is >= (c << 20) + add: add = 0
// gives the class boundaries, add = 0x100000 - kmin the first quartet of
// class c with fewer than kmin primitive quartets
__global__ void k_class_starts_f(const unsigned *__restrict__ keys, long long n, int ncls,
                                 unsigned add, long long *starts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ncls) return;
  long long lo = 0, hi = n;
  const unsigned key = ((unsigned)c << 20) + add;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  starts[c] = lo;
}

__global__ void k_symmetrize(const double *__restrict__ J, const double *__restrict__ K, int n,
                             double *G, bool accumulate) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int a = (int)(t / n), b = (int)(t % n);
  const long long tt = (long long)b * n + a;
  const double g = J[t] + J[tt] - 0.5 * (K[t] + K[tt]);
  G[t] = accumulate ? G[t] + g : g;
}

}  // namespace

void dens_max_device(MolCtx &m, const double *dP, cudaStream_t st) {
  k_dens_max<<<(m.nbas * m.nbas + 255) / 256, 256, 0, st>>>(dP, m.nao, m.aooff, m.nbas, m.Dsh);
  engine().launches++;
}

// ------------------------------------------------------------ context
static int mol_create_segmented(MolCtx &m, const int *atm, int natm, const int *bas, int nbas,
                                const double *env, long long nenv, cudaStream_t st);

// Generally contracted shells are split into segmented sub-shells first
// (gc_expand): the AO order is unchanged, so every matrix of the context is
// the one of the input basis.
int mol_create(MolCtx &m, const int *atm, int natm, const int *bas, int nbas, const double *env,
               long long nenv, cudaStream_t st) {
  GcExpanded x;
  if (int rc = gc_expand(bas, nbas, env, nenv, x)) return rc;
  if (!x.any) return mol_create_segmented(m, atm, natm, bas, nbas, env, nenv, st);
  m.gc = 1;
  return mol_create_segmented(m, atm, natm, x.bas.data(), (int)(x.bas.size() / 8), x.env.data(),
                              (long long)x.env.size(), st);
}

static int mol_create_segmented(MolCtx &m, const int *atm, int natm, const int *bas, int nbas,
                                const double *env, long long nenv, cudaStream_t st) {
  m.natm = natm; m.nbas = nbas; m.nenv = nenv;
  m.h_atm.assign(atm, atm + 6 * natm);
  m.h_bas.assign(bas, bas + 8 * nbas);
  m.h_env.assign(env, env + nenv);
  for (int s = 0; s < nbas; ++s) {
    const int *b = bas + 8 * s;
    if (b[1] < 0 || b[1] > ERI_LMAX || b[3] != 1 || b[2] < 1 || b[2] > ERI_KMAX)
      return set_error("molecule: shells must have l <= 3 and 1..31 primitives"),
             LRB_ERR_UNSUPPORTED;
    if (b[0] < 0 || b[0] >= natm || b[5] < 0 || b[6] < 0 || (long long)b[5] + b[2] > nenv ||
        (long long)b[6] + b[2] > nenv)
      return set_error("molecule: bas index out of range"), LRB_ERR_INPUT;
  }
  for (int a = 0; a < natm; ++a)
    if (atm[6 * a + 1] < 0 || (long long)atm[6 * a + 1] + 3 > nenv)
      return set_error("molecule: atm coordinate pointer out of range"), LRB_ERR_INPUT;
  m.h_aooff.assign(nbas + 1, 0);
  for (int s = 0; s < nbas; ++s) m.h_aooff[s + 1] = m.h_aooff[s] + ncart(bas[8 * s + 1]);
  m.nao = m.h_aooff[nbas];
  // pair table
  std::vector<PairInfo> pr;
  std::vector<int> pc;
  int npp = 0;
  for (int I = 0; I < nbas; ++I)
    for (int J = 0; J <= I; ++J) {
      int a = I, b = J;
      if (bas[8 * a + 1] < bas[8 * b + 1]) std::swap(a, b);
      PairInfo p;
      p.ish = a; p.jsh = b; p.pp_off = npp; p.npp = bas[8 * a + 2] * bas[8 * b + 2];
      npp += p.npp;
      pr.push_back(p);
      const int la = bas[8 * a + 1], lb = bas[8 * b + 1];
      pc.push_back(la * (la + 1) / 2 + lb);
    }
  m.npairs = (int)pr.size();
  m.npp = npp;
  m.h_pairs = pr;
  auto al = [&](void **p, size_t n) {
    return cudaMallocAsync(p, std::max(n, (size_t)16), st) == cudaSuccess;
  };
  if (!al((void **)&m.atm, sizeof(int) * 6 * natm) || !al((void **)&m.bas, sizeof(int) * 8 * nbas) ||
      !al((void **)&m.env, sizeof(double) * nenv) || !al((void **)&m.aooff, sizeof(int) * (nbas + 1)) ||
      !al((void **)&m.pairs, sizeof(PairInfo) * m.npairs) || !al((void **)&m.pcls, sizeof(int) * m.npairs) ||
      !al((void **)&m.pp, sizeof(PrimPair) * npp) || !al((void **)&m.Q, sizeof(double) * m.npairs) ||
      !al((void **)&m.Dsh, sizeof(double) * nbas * nbas) ||
      !al((void **)&m.centers, sizeof(double) * 3 * nbas))
    return set_error("molecule: device allocation failed"), LRB_ERR_ALLOC;
  FK_CK(cudaMemcpyAsync(m.atm, atm, sizeof(int) * 6 * natm, cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(m.bas, bas, sizeof(int) * 8 * nbas, cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(m.env, env, sizeof(double) * nenv, cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(m.aooff, m.h_aooff.data(), sizeof(int) * (nbas + 1), cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(m.pairs, pr.data(), sizeof(PairInfo) * m.npairs, cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(m.pcls, pc.data(), sizeof(int) * m.npairs, cudaMemcpyHostToDevice, st));
  {
    std::vector<double> cen(3 * (size_t)nbas);
    for (int s = 0; s < nbas; ++s)
      for (int d = 0; d < 3; ++d) cen[3 * s + d] = env[atm[6 * bas[8 * s] + 1] + d];
    FK_CK(cudaMemcpyAsync(m.centers, cen.data(), sizeof(double) * 3 * nbas, cudaMemcpyHostToDevice, st));
    FK_CK(cudaStreamSynchronize(st));   // cen goes out of scope
  }
  k_mol_pairs<<<(npp + 255) / 256, 256, 0, st>>>(m.pairs, m.npairs, m.atm, m.bas, m.env, m.pp, npp,
                                                  m.gc);
  engine().launches++;
  FK_CK(cudaGetLastError());
  // Schwarz factors from (IJ|IJ) cartesian blocks
  std::vector<int> quart(4 * (size_t)m.npairs), dims(2 * (size_t)m.npairs);
  std::vector<long long> boff(m.npairs + 1, 0);
  for (int p = 0; p < m.npairs; ++p) {
    const int I = pr[p].ish, J = pr[p].jsh;
    quart[4 * p] = I; quart[4 * p + 1] = J; quart[4 * p + 2] = I; quart[4 * p + 3] = J;
    const int ni = ncart(bas[8 * I + 1]), nj = ncart(bas[8 * J + 1]);
    dims[2 * p] = ni; dims[2 * p + 1] = nj;
    boff[p + 1] = boff[p] + (long long)ni * nj * ni * nj;
  }
  int *d_q = nullptr, *d_dims = nullptr;
  long long *d_boff = nullptr;
  double *d_blk = nullptr;
  if (!al((void **)&d_q, sizeof(int) * quart.size()) || !al((void **)&d_dims, sizeof(int) * dims.size()) ||
      !al((void **)&d_boff, sizeof(long long) * boff.size()) ||
      !al((void **)&d_blk, sizeof(double) * (size_t)boff[m.npairs]))
    return set_error("molecule: device allocation failed"), LRB_ERR_ALLOC;
  FK_CK(cudaMemcpyAsync(d_q, quart.data(), sizeof(int) * quart.size(), cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(d_dims, dims.data(), sizeof(int) * dims.size(), cudaMemcpyHostToDevice, st));
  FK_CK(cudaMemcpyAsync(d_boff, boff.data(), sizeof(long long) * boff.size(), cudaMemcpyHostToDevice, st));
  int rc = eri_batch_device(engine(), d_blk, 0, d_q, m.npairs, m.atm, natm, m.bas, nbas, m.env,
                            nenv, st, nullptr, nullptr, m.gc);
  if (rc) return rc;
  k_schwarz<<<(m.npairs + 255) / 256, 256, 0, st>>>(d_blk, d_boff, d_dims, m.npairs, m.Q);
  engine().launches++;
  FK_CK(cudaGetLastError());
  cudaFreeAsync(d_q, st);
  cudaFreeAsync(d_dims, st);
  cudaFreeAsync(d_boff, st);
  cudaFreeAsync(d_blk, st);
  FK_CK(cudaStreamSynchronize(st));
  // Schwarz factor of every primitive pair (the Fock builds' primitive
  // screening): (ij|ij) of single-primitive shells, in chunks of records
  // whose blocks take at most 256 MB
  {
    std::vector<int> pfirst(nbas + 1, 0);
    for (int sh = 0; sh < nbas; ++sh) pfirst[sh + 1] = pfirst[sh] + bas[8 * sh + 2];
    const int nps = pfirst[nbas];
    std::vector<int> pbas(8 * (size_t)nps);
    for (int sh = 0; sh < nbas; ++sh)
      for (int q = 0; q < bas[8 * sh + 2]; ++q) {
        int *r = &pbas[8 * (size_t)(pfirst[sh] + q)];
        const int *b = bas + 8 * sh;
        r[0] = b[0]; r[1] = b[1]; r[2] = 1; r[3] = 1; r[4] = b[4];
        r[5] = b[5] + q; r[6] = b[6] + q; r[7] = b[7] > 0 ? b[7] + q : 0;
      }
    std::vector<int> rq(4 * (size_t)npp), rdim(2 * (size_t)npp);
    for (int q = 0; q < m.npairs; ++q) {
      const int I = pr[q].ish, J = pr[q].jsh, ki = bas[8 * I + 2];
      for (int e = 0; e < pr[q].npp; ++e) {
        const int r = pr[q].pp_off + e;
        const int a = pfirst[I] + e % ki, b = pfirst[J] + e / ki;
        rq[4 * (size_t)r] = a; rq[4 * (size_t)r + 1] = b;
        rq[4 * (size_t)r + 2] = a; rq[4 * (size_t)r + 3] = b;
        rdim[2 * (size_t)r] = ncart(bas[8 * I + 1]);
        rdim[2 * (size_t)r + 1] = ncart(bas[8 * J + 1]);
      }
    }
    int *d_pbas = nullptr, *d_rq = nullptr, *d_rdim = nullptr;
    if (!al((void **)&m.lq, sizeof(float) * (size_t)npp) ||
        !al((void **)&d_pbas, sizeof(int) * pbas.size()) || !al((void **)&d_rq, sizeof(int) * rq.size()) ||
        !al((void **)&d_rdim, sizeof(int) * rdim.size()))
      return set_error("molecule: device allocation failed"), LRB_ERR_ALLOC;
    FK_CK(cudaMemcpyAsync(d_pbas, pbas.data(), sizeof(int) * pbas.size(), cudaMemcpyHostToDevice, st));
    FK_CK(cudaMemcpyAsync(d_rq, rq.data(), sizeof(int) * rq.size(), cudaMemcpyHostToDevice, st));
    FK_CK(cudaMemcpyAsync(d_rdim, rdim.data(), sizeof(int) * rdim.size(), cudaMemcpyHostToDevice, st));
    const long long cap = 256LL << 17;   // doubles of blocks per chunk (256 MB)
    for (int r0 = 0; r0 < npp;) {
      std::vector<long long> roff{0};
      int r1 = r0;
      while (r1 < npp) {
        const long long sz = (long long)rdim[2 * (size_t)r1] * rdim[2 * (size_t)r1 + 1];
        if (r1 > r0 && roff.back() + sz * sz > cap) break;
        roff.push_back(roff.back() + sz * sz);
        ++r1;
      }
      long long *d_roff = nullptr;
      double *d_pb = nullptr;
      if (!al((void **)&d_roff, sizeof(long long) * roff.size()) ||
          !al((void **)&d_pb, sizeof(double) * (size_t)roff.back()))
        return set_error("molecule: device allocation failed"), LRB_ERR_ALLOC;
      FK_CK(cudaMemcpyAsync(d_roff, roff.data(), sizeof(long long) * roff.size(),
                            cudaMemcpyHostToDevice, st));
      int rc2 = eri_batch_device(engine(), d_pb, 0, d_rq + 4 * (size_t)r0, r1 - r0, m.atm, natm,
                                 d_pbas, nps, m.env, nenv, st, nullptr, nullptr, m.gc);
      if (rc2) return rc2;
      k_prim_schwarz<<<(r1 - r0 + 255) / 256, 256, 0, st>>>(d_pb, d_roff, d_rdim + 2 * (size_t)r0,
                                                             r1 - r0, m.lq + r0);
      engine().launches++;
      FK_CK(cudaGetLastError());
      cudaFreeAsync(d_roff, st);
      cudaFreeAsync(d_pb, st);
      FK_CK(cudaStreamSynchronize(st));   // roff goes out of scope
      r0 = r1;
    }
    cudaFreeAsync(d_pbas, st);
    cudaFreeAsync(d_rq, st);
    cudaFreeAsync(d_rdim, st);
    FK_CK(cudaStreamSynchronize(st));
  }
  // pairs by descending Schwarz factor, for the candidate enumeration
  {
    std::vector<double> q(m.npairs);
    FK_CK(cudaMemcpy(q.data(), m.Q, sizeof(double) * m.npairs, cudaMemcpyDeviceToHost));
    std::vector<int> ord(m.npairs);
    for (int p = 0; p < m.npairs; ++p) ord[p] = p;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return q[a] > q[b]; });
    std::vector<double> qs(m.npairs);
    for (int p = 0; p < m.npairs; ++p) qs[p] = q[ord[p]];
    if (!al((void **)&m.qorder, sizeof(int) * m.npairs) || !al((void **)&m.Qs, sizeof(double) * m.npairs) ||
        !al((void **)&m.qcnt, sizeof(int) * m.npairs) ||
        !al((void **)&m.qoff, sizeof(long long) * (m.npairs + 1)) || !al((void **)&m.dmax, sizeof(double)))
      return set_error("molecule: device allocation failed"), LRB_ERR_ALLOC;
    FK_CK(cudaMemcpyAsync(m.qorder, ord.data(), sizeof(int) * m.npairs, cudaMemcpyHostToDevice, st));
    FK_CK(cudaMemcpyAsync(m.Qs, qs.data(), sizeof(double) * m.npairs, cudaMemcpyHostToDevice, st));
    FK_CK(cudaStreamSynchronize(st));
  }
  return LRB_OK;
}

void mol_destroy(MolCtx &m, cudaStream_t st) {
  for (void *p : {(void *)m.atm, (void *)m.bas, (void *)m.env, (void *)m.aooff, (void *)m.pairs,
                  (void *)m.pcls, (void *)m.pp, (void *)m.Q, (void *)m.Dsh, (void *)m.centers,
                  (void *)m.qorder, (void *)m.Qs, (void *)m.qcnt, (void *)m.qoff, (void *)m.dmax,
                  (void *)m.lq})
    if (p) cudaFreeAsync(p, st);
  cudaStreamSynchronize(st);
}

// ------------------------------------------------------------ build
int fock_build(MolCtx &m, const double *dP, double *dG, double tau, cudaStream_t st,
               FockStats *stats, int prec, double tau32, bool accumulate, int rank, int nranks) {
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return set_error("fock: need 0 <= rank < nranks"), LRB_ERR_INPUT;
  Engine &eng = engine();
  const ClassEntry *tab = class_table();
  if (!tab) return LRB_ERR_CUDA;
  const int n = m.nao, nbas = m.nbas;
  // candidates: sorted positions i >= j with Q_i Q_j 2 max|D| >= tau
  k_dens_max<<<(nbas * nbas + 255) / 256, 256, 0, st>>>(dP, n, m.aooff, nbas, m.Dsh);
  k_max_reduce<<<1, 1024, 0, st>>>(m.Dsh, nbas * nbas, m.dmax);
  k_cand_count<<<(m.npairs + 255) / 256, 256, 0, st>>>(m.Qs, m.npairs, m.dmax, tau, m.qcnt);
  eng.launches += 3;
  {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, m.qcnt, m.qoff, m.npairs + 1, st);
    void *tmp = eng.ws.reserve_aux(st, tb + 64);
    if (!tmp) return set_error("fock: workspace allocation failed"), LRB_ERR_ALLOC;
    // qcnt has npairs entries; the scan of npairs + 1 reads one past it, so
    // run it on npairs and add the last count on the host
    FK_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, m.qcnt, m.qoff, m.npairs, st));
  }
  long long ncand = 0;
  {
    long long lastoff = 0;
    int lastcnt = 0;
    FK_CK(cudaMemcpyAsync(&lastoff, m.qoff + m.npairs - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    FK_CK(cudaMemcpyAsync(&lastcnt, m.qcnt + m.npairs - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    FK_CK(cudaStreamSynchronize(st));
    ncand = lastoff + lastcnt;
  }
  // job capacity: all candidates (worst case, nothing screened further)
  const size_t cap = (size_t)std::max(ncand, 1LL);
  const size_t need = carve_size(sizeof(int2) * cap) + 2 * carve_size(sizeof(unsigned) * cap) +
                      2 * carve_size(sizeof(int) * cap) + 2 * carve_size(sizeof(double) * (size_t)n * n) +
                      carve_size(sizeof(long long) * 256) + carve_size(sizeof(unsigned long long)) +
                      carve_size(sizeof(int) * 256);
  char *base = eng.ws.reserve_extra(st, need) ? (char *)eng.ws.extra.ptr : nullptr;
  if (!base) return set_error("fock: workspace allocation failed"), LRB_ERR_ALLOC;
  Carver cv(base);
  int2 *jobs = cv.take<int2>(cap);
  unsigned *keys = cv.take<unsigned>(cap), *keys2 = cv.take<unsigned>(cap);
  int *idx = cv.take<int>(cap), *idx2 = cv.take<int>(cap);
  double *J = cv.take<double>((size_t)n * n), *K = cv.take<double>((size_t)n * n);
  long long *starts = cv.take<long long>(256);
  unsigned long long *count = cv.take<unsigned long long>(1);
  int *counters = cv.take<int>(256);   // task counters: slot kernels, then lane kernels
  FK_CK(cudaMemsetAsync(J, 0, sizeof(double) * (size_t)n * n, st));
  FK_CK(cudaMemsetAsync(K, 0, sizeof(double) * (size_t)n * n, st));
  FK_CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
  FK_CK(cudaMemsetAsync(counters, 0, sizeof(int) * 256, st));
  if (ncand > 0) {
    k_screen_sorted<<<(unsigned)((ncand + 255) / 256), 256, 0, st>>>(
        m.pairs, m.pcls, m.Q, m.qorder, m.qoff, m.npairs, m.Dsh, nbas, ncand, tau, prec, tau32,
        rank, nranks, jobs, keys, idx, count, cap);
    ++eng.launches;
  }
  FK_CK(cudaGetLastError());
  unsigned long long nj = 0;
  long long n32 = 0;
  FK_CK(cudaMemcpyAsync(&nj, count, sizeof(nj), cudaMemcpyDeviceToHost, st));
  FK_CK(cudaStreamSynchronize(st));
  if (nj > cap) nj = cap;
  if (nj > 0) {
    size_t tmpb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys, keys2, idx, idx2, (int)nj, 0, 32, st);
    void *tmp = eng.ws.reserve_aux(st, tmpb + 64);
    if (!tmp) return set_error("fock: workspace allocation failed"), LRB_ERR_ALLOC;
    FK_CK(cub::DeviceRadixSort::SortPairs(tmp, tmpb, keys, keys2, idx, idx2, (int)nj, 0, 32, st));
    static_assert(2 * NCLASS + 1 <= 128, "class starts launch covers 128 ids");
    k_class_starts_f<<<1, 128, 0, st>>>(keys2, (long long)nj, 2 * NCLASS, 0u, starts);
    // within a class the keys run by decreasing primitive-quartet count: the
    // quartets with at least lp_min of them come first and go to the
    // lane-per-primitive kernel where the class has one
    const int lp_min = fock_lp_min();
    k_class_starts_f<<<1, 128, 0, st>>>(keys2, (long long)nj, 2 * NCLASS,
                                        0x100000u - (unsigned)lp_min, starts + 128);
    eng.launches += 2;
    long long cls_begin[256];
    FK_CK(cudaMemcpyAsync(cls_begin, starts, sizeof(long long) * 256, cudaMemcpyDeviceToHost, st));
    FK_CK(cudaStreamSynchronize(st));
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const double *rys = rys_table_device();
    EriParams prm{};
    prm.pp = m.pp;
    prm.centers = m.centers;
    prm.expcutoff = m.h_env[0] == 0.0 ? eng.expcutoff : std::max(40.0, m.h_env[0]) + 1.0;
    prm.omega = m.nenv > 8 ? m.h_env[8] : 0.0;
    prm.sph = 0;
    FockParams fk;
    fk.jobs = jobs;
    fk.pairs = m.pairs;
    fk.aooff = m.aooff;
    fk.P = dP;
    fk.J = J;
    fk.K = K;
    fk.n = n;
    fk.prim_count = nullptr;
    // primitive screening: the FP64 quartets at the context's threshold, the
    // FP32 ones at the larger of it and the build's quartet threshold
    const double tprim = m.tau_prim > 0.0 ? (prec == 1 ? std::max(m.tau_prim, tau) : m.tau_prim) : 0.0;
    fk.lq = tprim > 0.0 ? m.lq : nullptr;
    fk.tau_prim = tprim;
    fk.Dsh = m.Dsh;
    fk.nbas = nbas;
    if (eng.profile && !eng.fock_prim) {
      if (cudaMalloc((void **)&eng.fock_prim, 128 * sizeof(unsigned long long)) != cudaSuccess)
        return set_error("fock: counter allocation failed"), LRB_ERR_ALLOC;
      FK_CK(cudaMemset(eng.fock_prim, 0, 128 * sizeof(unsigned long long)));
    }
    for (int cc = 0; cc < 2 * NCLASS; ++cc) {
      long long b0 = cls_begin[cc];
      const long long b1 = cls_begin[cc + 1];
      if (b1 <= b0) continue;
      const int c = cc % NCLASS, fi = cc < NCLASS ? 1 : 2;
      if (fi == 2) n32 += b1 - b0;
      const ClassEntry &ce = tab[c];
      ProfRecord rec{cc, nullptr, nullptr};
      if (eng.profile) {
        cudaEventCreate(&rec.start);
        cudaEventCreate(&rec.stop);
        cudaEventRecord(rec.start, st);
        fk.prim_count = eng.fock_prim + cc;
        eng.fock_quartets[cc] += b1 - b0;
      } else {
        fk.prim_count = nullptr;
      }
      const long long split = std::min(std::max(cls_begin[128 + cc], b0), b1);
      if (ce.lp[fi - 1] && split > b0) {
        // one warp per shell quartet, one lane per primitive quartet
        const EriKernelFn lp = ce.lp[fi - 1];
        prm.order = idx2 + b0;
        prm.njobs = (int)(split - b0);
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lp, ERI_THREADS, ce.lp_smem[fi - 1]);
        if (per_sm < 1) per_sm = 1;
        long long grid = (long long)nsm * per_sm;
        const long long needg = (prm.njobs + ERI_WARPS - 1) / ERI_WARPS;
        if (grid > needg) grid = needg;
        lp<<<(unsigned)grid, ERI_THREADS, ce.lp_smem[fi - 1], st>>>(
            prm, fk, rys + RYS_TAB_OFFSET[ce.nr], counters + 128 + cc);
        FK_CK(cudaGetLastError());
        eng.launches++;
        b0 = split;
      }
      if (b1 > b0) {
        prm.order = idx2 + b0;
        prm.njobs = (int)(b1 - b0);
        int per_sm = 0;
        if (ce.gen)
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gen_kernel(1), GEN_THREADS, ce.smem[1]);
        else
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ce.fn[fi], ERI_THREADS, ce.smem[fi]);
        if (per_sm < 1) per_sm = 1;
        const long long tasks = (prm.njobs + ce.slots - 1) / ce.slots;
        long long grid = (long long)nsm * per_sm;
        const long long needg = ce.gen ? tasks : (tasks + ERI_WARPS - 1) / ERI_WARPS;
        if (grid > needg) grid = needg;
        if (ce.gen)
          gen_kernel(1)<<<(unsigned)grid, GEN_THREADS, ce.smem[1], st>>>(
              prm, fk, ce.g, rys + RYS_TAB_OFFSET[ce.nr], counters + cc);
        else
          ce.fn[fi]<<<(unsigned)grid, ERI_THREADS, ce.smem[fi], st>>>(
              prm, fk, rys + RYS_TAB_OFFSET[ce.nr], counters + cc);
        FK_CK(cudaGetLastError());
        eng.launches++;
      }
      if (eng.profile) {
        cudaEventRecord(rec.stop, st);
        eng.prof.push_back(rec);
      }
    }
  }
  k_symmetrize<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, st>>>(J, K, n, dG, accumulate);
  eng.launches++;
  FK_CK(cudaGetLastError());
  if (stats) {
    stats->candidates = ncand;
    stats->quartets = (long long)nj;
    stats->fp32_quartets = n32;
  }
  return LRB_OK;
}

}  // namespace lrb

// Minimum primitive-quartet count of the lane-per-primitive Fock kernels;
// kmin > 0 sets it (0x100000 or more: never), kmin <= 0 only reads it.
LRB_API int lrb_fock_lane_min(int kmin) {
  if (kmin > 0) lrb::g_lp_min.store(std::min(kmin, 0x100000));
  return lrb::fock_lp_min();
}
