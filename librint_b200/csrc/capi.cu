// C ABI of librint_b200: batched ERIs, the libcint int2e_* entry points and
// librint's p2c.rs-shaped functions.  Every compute path runs on the GPU;
// there is no CPU fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "batch_plan.h"
#include "engine.h"
#include "eri_device.cuh"
#include "fock.h"
#include "grad.h"

using namespace lrb;

namespace {

#define CK(x)                                  \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) {                   \
      set_error(cudaGetErrorString(e_));       \
      return LRB_ERR_CUDA;                     \
    }                                          \
  } while (0)

// Device copies of one molecule's atm/bas/env.
struct DevMol {
  int *atm = nullptr, *bas = nullptr;
  double *env = nullptr;
  int natm = 0, nbas = 0;
  long long nenv = 0;
  int upload(cudaStream_t st, const int *a, int na, const int *b, int nb, const double *e,
             long long ne) {
    natm = na; nbas = nb; nenv = ne;
    CK(cudaMallocAsync((void **)&atm, sizeof(int) * 6 * (size_t)std::max(na, 1), st));
    CK(cudaMallocAsync((void **)&bas, sizeof(int) * 8 * (size_t)std::max(nb, 1), st));
    CK(cudaMallocAsync((void **)&env, sizeof(double) * (size_t)std::max(ne, 1LL), st));
    CK(cudaMemcpyAsync(atm, a, sizeof(int) * 6 * (size_t)na, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(bas, b, sizeof(int) * 8 * (size_t)nb, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env, e, sizeof(double) * (size_t)ne, cudaMemcpyHostToDevice, st));
    return LRB_OK;
  }
  // device arrays only; the caller fills them
  int alloc(cudaStream_t st, int na, int nb, long long ne) {
    natm = na; nbas = nb; nenv = ne;
    CK(cudaMallocAsync((void **)&atm, sizeof(int) * 6 * (size_t)std::max(na, 1), st));
    CK(cudaMallocAsync((void **)&bas, sizeof(int) * 8 * (size_t)std::max(nb, 1), st));
    CK(cudaMallocAsync((void **)&env, sizeof(double) * (size_t)std::max(ne, 1LL), st));
    return LRB_OK;
  }
  void release(cudaStream_t st) {
    if (atm) cudaFreeAsync(atm, st);
    if (bas) cudaFreeAsync(bas, st);
    if (env) cudaFreeAsync(env, st);
    atm = bas = nullptr;
    env = nullptr;
  }
};

// env length implied by atm/bas (the libcint ABI passes no env length).
long long env_extent(const int *atm, int natm, const int *bas, int nbas) {
  long long n = 9;   // env[0..8] are read (expcutoff, omega)
  for (int a = 0; a < natm; ++a) {
    n = std::max(n, (long long)atm[6 * a + 1] + 3);
    if (atm[6 * a + 2] == 2) n = std::max(n, (long long)atm[6 * a + 3] + 1);
  }
  for (int s = 0; s < nbas; ++s) {
    const int *b = bas + 8 * s;
    n = std::max(n, (long long)b[5] + b[2]);
    n = std::max(n, (long long)b[6] + (long long)b[2] * b[3]);
  }
  return n;
}

int shell_dim(int coord, const int *bas, int s) {
  const int l = bas[8 * s + 1];
  return (coord == 0 ? ncart(l) : nsph(l)) * bas[8 * s + 3];
}

int check_common(const int *atm, int natm, const int *bas, int nbas, const double *env,
                 long long nenv) {
  if (!atm || !bas || !env || natm <= 0 || nbas <= 0 || nenv <= 0)
    return set_error("empty or NULL atm/bas/env"), LRB_ERR_INPUT;
  return LRB_OK;
}

// Two device buffers of na and nb doubles on st; on failure neither is
// kept and the allocation error is cleared.
int alloc_pair(cudaStream_t st, size_t na, double **a, size_t nb, double **b) {
  *a = *b = nullptr;
  if (cudaMallocAsync((void **)a, std::max(na, (size_t)1) * 8, st) != cudaSuccess) {
    *a = nullptr;
  } else if (cudaMallocAsync((void **)b, std::max(nb, (size_t)1) * 8, st) != cudaSuccess) {
    *b = nullptr;
  }
  if (*a && *b) return LRB_OK;
  cudaGetLastError();
  if (*a) cudaFreeAsync(*a, st);
  *a = *b = nullptr;
  return set_error("device allocation failed"), LRB_ERR_ALLOC;
}

// Dense symmetric tensor from canonical quartet blocks.
__global__ void k_scatter8(const double *__restrict__ blocks, const long long *__restrict__ boff,
                           const int *__restrict__ quart, const int *__restrict__ aooff,
                           const int *__restrict__ dim, int nq, long long n, double *R) {
  const int q = blockIdx.x;
  if (q >= nq) return;
  const int i = quart[4 * q], j = quart[4 * q + 1], k = quart[4 * q + 2], l = quart[4 * q + 3];
  const int di = dim[i], dj = dim[j], dk = dim[k], dl = dim[l];
  const int tot = di * dj * dk * dl;
  const double *b = blocks + boff[q];
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    int t = e;
    const int a = t % di; t /= di;
    const int bb = t % dj; t /= dj;
    const int c = t % dk;
    const int d = t / dk;
    const long long A = aooff[i] + a, B = aooff[j] + bb, Cc = aooff[k] + c, D = aooff[l] + d;
    const double v = b[e];
    R[((A * n + B) * n + Cc) * n + D] = v;
    R[((B * n + A) * n + Cc) * n + D] = v;
    R[((A * n + B) * n + D) * n + Cc] = v;
    R[((B * n + A) * n + D) * n + Cc] = v;
    R[((Cc * n + D) * n + A) * n + B] = v;
    R[((D * n + Cc) * n + A) * n + B] = v;
    R[((Cc * n + D) * n + B) * n + A] = v;
    R[((D * n + Cc) * n + B) * n + A] = v;
  }
}

}  // namespace

struct LrbCintOpt {
  DevMol mol;
  const int *h_atm = nullptr, *h_bas = nullptr;
  const double *h_env = nullptr;
};

extern "C" {

long long lrb_int2e_batch_len(int coord, const int *shls, long long nq, const int *bas, int nbas) {
  if (!shls || !bas || nq < 0) return -1;
  // per host-thread part: -1 on a shell index out of range, else its length
  long long part[64] = {0};   // host_parallel runs at most 32 parts
  std::atomic<int> slot{0};
  std::atomic<bool> bad{false};
  plan::host_parallel(nq, plan::HOST_GRAIN, [&](long long b, long long e) {
    for (long long q = 4 * b; q < 4 * e; ++q)
      if (shls[q] < 0 || shls[q] >= nbas) {
        bad.store(true, std::memory_order_relaxed);
        return;
      }
    part[(size_t)slot.fetch_add(1)] = eri_batch_out_len(coord, shls + 4 * b, e - b, bas);
  });
  if (bad.load()) return -1;
  long long n = 0;
  for (long long v : part) n += v;
  return n;
}

int lrb_int2e_batch_device(double *out, int coord, const int *shls, long long nq,
                           const int *atm, int natm, const int *bas, int nbas,
                           const double *env, long long nenv, void *stream) {
  if (nq == 0) return LRB_OK;
  if (!out || !shls || nq < 0) return set_error("bad output or quartet list"), LRB_ERR_INPUT;
  return eri_batch_device(engine(), out, coord, shls, nq, atm, natm, bas, nbas, env, nenv,
                          (cudaStream_t)stream, nullptr);
}

// Chunk limits: at most CHUNK_Q quartets and, past a chunk's first quartet,
// CHUNK_OUT output doubles (256 MB); env[0..ENV_HEAD) holds the settings
// every chunk reads (cutoff, omega).
constexpr long long CHUNK_Q = 1 << 18, CHUNK_OUT = 1 << 25, ENV_HEAD = 20;

// Host buffers in and out.  The quartets run in chunks through three
// non-blocking streams: copies in (the chunk's quartet list, and in the
// streamed layout its part of the molecule), kernels, copies out.  Chunk c
// uses device slot c % 2 for its quartet list and output, so chunk c+1's
// copy in and chunk c-1's copy out overlap chunk c's kernels; events hand
// each slot on (copy in -> kernels -> copy out -> the copy in two chunks
// later).  The kernels of all chunks share the engine's workspace and run in
// order on the one kernel stream.  The batch has been checked and planned by
// plan::plan_batch.
static int batch_host(double *out, int coord, const int *shls, const int *atm, int natm,
                      const int *bas, int nbas, const double *env, long long nenv, int gc_screen,
                      const plan::BatchPlan &p) {
  int rc = LRB_OK;
  const std::vector<long long> &qb = p.qb, &ob = p.ob;
  const long long max_q = p.max_q, max_len = p.max_len;
  const int nchunk = p.nchunk();
  const long long head = std::min(nenv, ENV_HEAD);
  const std::vector<plan::ChunkRange> &rg = p.rg;
  const bool streamed = p.streamed;

  Engine &eng = engine();
  for (int i = 0; i < 3; ++i)
    if (!eng.pipe[i] && cudaStreamCreateWithFlags(&eng.pipe[i], cudaStreamNonBlocking) != cudaSuccess)
      return set_error("stream creation failed"), LRB_ERR_CUDA;
  for (int i = 0; i < 2; ++i)
    for (cudaEvent_t *ev : {&eng.ev_in[i], &eng.ev_cmp[i], &eng.ev_out[i]})
      if (!*ev && cudaEventCreateWithFlags(ev, cudaEventDisableTiming) != cudaSuccess)
        return set_error("event creation failed"), LRB_ERR_CUDA;
  cudaStream_t s_in = eng.pipe[0], s_k = eng.pipe[1], s_out = eng.pipe[2];
  // every device buffer of the call is allocated on the kernel stream before
  // the synchronisation below, so all three streams may use it afterwards
  DevMol m;
  double *cen = (double *)eng.pipe_centers.get(s_k, sizeof(double) * 3 * (size_t)nbas + 256);
  bool got = cen != nullptr;
  for (int X = 0; X < std::min(nchunk, 2); ++X)
    got = got && eng.pipe_in[X].get(s_k, sizeof(int) * 4 * (size_t)max_q) &&
          eng.pipe_out[X].get(s_k, sizeof(double) * (size_t)max_len);
  if (!got) return set_error("device allocation failed"), LRB_ERR_ALLOC;
  int *d_err = reinterpret_cast<int *>(cen + 3 * (size_t)nbas);
  if (!streamed) {
    // the whole molecule, and shell centres once per call (synchronises s_k)
    rc = m.upload(s_k, atm, natm, bas, nbas, env, nenv);
    if (!rc) rc = eri_centers(m.atm, natm, m.bas, nbas, m.env, nenv, cen, d_err, s_k);
  } else {
    // device arrays of full size; each chunk fills its own ranges
    rc = m.alloc(s_k, natm, nbas, nenv);
    if (!rc && (cudaMemcpyAsync(m.env, env, sizeof(double) * head, cudaMemcpyHostToDevice, s_k) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s_k) != cudaSuccess))
      rc = (set_error("copy failed"), LRB_ERR_CUDA);
  }
  for (int c = 0; c < nchunk && !rc; ++c) {
    const int X = c & 1;
    const long long nqc = qb[c + 1] - qb[c], len = ob[c + 1] - ob[c];
    int *d_sh = (int *)eng.pipe_in[X].ptr;
    double *d_o = (double *)eng.pipe_out[X].ptr;
    // copy in: slot X's quartet list is free once chunk c-2's kernels ran
    bool ok = c < 2 || cudaStreamWaitEvent(s_in, eng.ev_cmp[X], 0) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_sh, shls + 4 * qb[c], sizeof(int) * 4 * (size_t)nqc,
                               cudaMemcpyHostToDevice, s_in) == cudaSuccess;
    if (streamed) {
      const plan::ChunkRange &r = rg[c];
      ok = ok && cudaMemcpyAsync(m.bas + 8 * (size_t)r.s0, bas + 8 * (size_t)r.s0,
                                 sizeof(int) * 8 * (size_t)(r.s1 - r.s0), cudaMemcpyHostToDevice,
                                 s_in) == cudaSuccess;
      ok = ok && cudaMemcpyAsync(m.atm + 6 * (size_t)r.a0, atm + 6 * (size_t)r.a0,
                                 sizeof(int) * 6 * (size_t)(r.a1 - r.a0), cudaMemcpyHostToDevice,
                                 s_in) == cudaSuccess;
      ok = ok && cudaMemcpyAsync(m.env + r.e0, env + r.e0, sizeof(double) * (size_t)(r.e1 - r.e0),
                                 cudaMemcpyHostToDevice, s_in) == cudaSuccess;
    }
    ok = ok && cudaEventRecord(eng.ev_in[X], s_in) == cudaSuccess;
    // kernels: after this chunk's copy in, and after chunk c-2's output left slot X
    ok = ok && cudaStreamWaitEvent(s_k, eng.ev_in[X], 0) == cudaSuccess;
    ok = ok && (c < 2 || cudaStreamWaitEvent(s_k, eng.ev_out[X], 0) == cudaSuccess);
    if (!ok) {
      rc = (set_error("copy failed"), LRB_ERR_CUDA);
      break;
    }
    if (streamed)
      eri_centers_async(m.atm, natm, m.bas + 8 * (size_t)rg[c].s0, rg[c].s1 - rg[c].s0, m.env,
                        nenv, cen + 3 * (size_t)rg[c].s0, d_err, s_k);
    rc = eri_batch_device(eng, d_o, coord, d_sh, nqc, m.atm, natm, m.bas, nbas, m.env, nenv, s_k,
                          nullptr, cen, gc_screen);
    if (rc) break;
    // copy out, after the chunk's kernels
    if (cudaEventRecord(eng.ev_cmp[X], s_k) != cudaSuccess ||
        cudaStreamWaitEvent(s_out, eng.ev_cmp[X], 0) != cudaSuccess ||
        cudaMemcpyAsync(out + ob[c], d_o, sizeof(double) * (size_t)len, cudaMemcpyDeviceToHost,
                        s_out) != cudaSuccess ||
        cudaEventRecord(eng.ev_out[X], s_out) != cudaSuccess)
      rc = (set_error("copy failed"), LRB_ERR_CUDA);
  }
  cudaError_t e = cudaSuccess;
  for (cudaStream_t s : {s_in, s_k, s_out}) {
    const cudaError_t ei = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = ei;
  }
  m.release(s_k);
  const cudaError_t ef = cudaStreamSynchronize(s_k);
  if (e == cudaSuccess) e = ef;
  if (!rc && e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    rc = LRB_ERR_CUDA;
  }
  return rc;
}

static int int2e_batch_host(double *out, int coord, const int *shls, long long nq,
                            const int *atm, int natm, const int *bas, int nbas, const double *env,
                            long long nenv);

int lrb_int2e_batch(double *out, int coord, const int *shls, long long nq, const int *atm,
                    int natm, const int *bas, int nbas, const double *env, long long nenv) {
  // host memory for the plan and the generally contracted split may run out;
  // no exception leaves the C ABI
  try {
    return int2e_batch_host(out, coord, shls, nq, atm, natm, bas, nbas, env, nenv);
  } catch (const std::bad_alloc &) {
    return set_error("host allocation failed"), LRB_ERR_ALLOC;
  } catch (...) {
    return set_error("host error"), LRB_ERR_INPUT;
  }
}

static int int2e_batch_host(double *out, int coord, const int *shls, long long nq,
                            const int *atm, int natm, const int *bas, int nbas, const double *env,
                            long long nenv) {
  if (nq == 0) return LRB_OK;
  if (!out || !shls || nq < 0) return set_error("bad output or quartet list"), LRB_ERR_INPUT;
  int rc = check_common(atm, natm, bas, nbas, env, nenv);
  if (rc) return rc;
  if (coord != 0 && coord != 1) return set_error("coord must be 0 or 1"), LRB_ERR_INPUT;
  // every check before any device work, chunks and molecule ranges, on the
  // host threads; gc_expand runs only when a shell has nctr > 1
  plan::BatchPlan p;
  const char *msg = "";
  if ((rc = plan::plan_batch(coord, shls, nq, atm, natm, bas, nbas, nenv, std::min(nenv, ENV_HEAD),
                             CHUNK_Q, CHUNK_OUT, p, &msg)))
    return set_error(msg), rc;
  if (!p.gc) return batch_host(out, coord, shls, atm, natm, bas, nbas, env, nenv, 0, p);
  GcExpanded x;
  if ((rc = gc_expand(bas, nbas, env, nenv, x))) return rc;
  // Generally contracted shells: every quartet becomes prod(nctr) quartets of
  // segmented sub-shells (contraction of i fastest), computed as one batch
  // and placed into the quartet's block at rows ctr * nf + component
  // (libcint's layout of a shell with several contractions).
  std::vector<int> sub;
  for (long long q = 0; q < nq; ++q) {
    const int *s4 = shls + 4 * q;
    const int nc[4] = {bas[8 * s4[0] + 3], bas[8 * s4[1] + 3], bas[8 * s4[2] + 3], bas[8 * s4[3] + 3]};
    for (int cl = 0; cl < nc[3]; ++cl)
      for (int ck = 0; ck < nc[2]; ++ck)
        for (int cj = 0; cj < nc[1]; ++cj)
          for (int ci = 0; ci < nc[0]; ++ci) {
            const int t[4] = {x.first[s4[0]] + ci, x.first[s4[1]] + cj, x.first[s4[2]] + ck,
                              x.first[s4[3]] + cl};
            sub.insert(sub.end(), t, t + 4);
          }
  }
  const long long nsub = (long long)sub.size() / 4;
  const int nbx = (int)(x.bas.size() / 8);
  const long long nenx = (long long)x.env.size();
  plan::BatchPlan px;
  if ((rc = plan::plan_batch(coord, sub.data(), nsub, atm, natm, x.bas.data(), nbx, nenx,
                             std::min(nenx, ENV_HEAD), CHUNK_Q, CHUNK_OUT, px, &msg)))
    return set_error(msg), rc;
  // the sub-shells' screening coefficients (bas slot 7) sit at the end of the
  // expanded env, outside every chunk's env range: upload the whole molecule
  px.streamed = false;
  std::vector<double> tmp((size_t)eri_batch_out_len(coord, sub.data(), nsub, x.bas.data()));
  rc = batch_host(tmp.data(), coord, sub.data(), atm, natm, x.bas.data(), nbx, x.env.data(), nenx,
                  1, px);
  if (rc) return rc;
  size_t src = 0, dst = 0;
  for (long long q = 0; q < nq; ++q) {
    const int *s4 = shls + 4 * q;
    int nf[4], nc[4], N[4];
    for (int a = 0; a < 4; ++a) {
      const int l = bas[8 * s4[a] + 1];
      nf[a] = coord == 0 ? ncart(l) : nsph(l);
      nc[a] = bas[8 * s4[a] + 3];
      N[a] = nf[a] * nc[a];
    }
    for (int cl = 0; cl < nc[3]; ++cl)
      for (int ck = 0; ck < nc[2]; ++ck)
        for (int cj = 0; cj < nc[1]; ++cj)
          for (int ci = 0; ci < nc[0]; ++ci)
            for (int d = 0; d < nf[3]; ++d)
              for (int c = 0; c < nf[2]; ++c)
                for (int b = 0; b < nf[1]; ++b)
                  for (int a = 0; a < nf[0]; ++a)
                    out[dst + (ci * nf[0] + a) +
                        (size_t)N[0] * ((cj * nf[1] + b) +
                                        (size_t)N[1] * ((ck * nf[2] + c) + (size_t)N[2] * (cl * nf[3] + d)))] =
                        tmp[src++];
    dst += (size_t)N[0] * N[1] * N[2] * N[3];
  }
  return LRB_OK;
}

// ------------------------------------------------------------ libcint ABI
static int int2e_one(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                     double *env, CINTOpt *opt, int coord) {
  int d[4];
  for (int a = 0; a < 4; ++a) {
    if (shls[a] < 0 || shls[a] >= nbas) return set_error("shell index out of range"), -1;
    d[a] = shell_dim(coord, bas, shls[a]);
  }
  const long long blk = (long long)d[0] * d[1] * d[2] * d[3];
  if (!out) return (int)blk;
  bool gc = false;
  for (int a = 0; a < 4; ++a) gc = gc || bas[8 * shls[a] + 3] > 1;
  cudaStream_t st = nullptr;
  DevMol local;
  const DevMol *m = nullptr;
  if (opt && opt->h_atm == atm && opt->h_bas == bas && opt->h_env == env) {
    m = &opt->mol;
  } else {
    const long long nenv = env_extent(atm, natm, bas, nbas);
    if (check_common(atm, natm, bas, nbas, env, nenv)) return -1;
    if (local.upload(st, atm, natm, bas, nbas, env, nenv)) return -1;
    m = &local;
  }
  int *d_sh = nullptr;
  double *d_out = nullptr;
  std::vector<double> blkbuf(blk);
  int rc = 0;
  if (gc) {
    // generally contracted shells go through the host batch path
    rc = lrb_int2e_batch(blkbuf.data(), coord, shls, 1, atm, natm, bas, nbas, env,
                         env_extent(atm, natm, bas, nbas));
  } else if (cudaMallocAsync((void **)&d_sh, 4 * sizeof(int), st) != cudaSuccess ||
      cudaMallocAsync((void **)&d_out, sizeof(double) * blk, st) != cudaSuccess) {
    rc = -1;
  } else {
    cudaMemcpyAsync(d_sh, shls, 4 * sizeof(int), cudaMemcpyHostToDevice, st);
    rc = eri_batch_device(engine(), d_out, coord, d_sh, 1, m->atm, m->natm, m->bas, m->nbas,
                          m->env, m->nenv, st, nullptr);
    if (!rc) cudaMemcpyAsync(blkbuf.data(), d_out, sizeof(double) * blk, cudaMemcpyDeviceToHost, st);
  }
  if (d_sh) cudaFreeAsync(d_sh, st);
  if (d_out) cudaFreeAsync(d_out, st);
  if (m == &local) local.release(st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
  if (rc) {
    // reference behaviour on failure: zero block, 0 returned
    if (!dims) std::memset(out, 0, sizeof(double) * blk);
    return 0;
  }
  int nz = 0;
  for (long long e = 0; e < blk; ++e) nz |= blkbuf[e] != 0.0;
  if (!dims) {
    std::memcpy(out, blkbuf.data(), sizeof(double) * blk);
  } else {
    long long e = 0;
    for (int l = 0; l < d[3]; ++l)
      for (int k = 0; k < d[2]; ++k)
        for (int j = 0; j < d[1]; ++j)
          for (int i = 0; i < d[0]; ++i, ++e)
            out[i + (long long)dims[0] * (j + (long long)dims[1] * (k + (long long)dims[2] * l))] = blkbuf[e];
  }
  return nz;
}

int int2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
              double *env, CINTOpt *opt, double *cache) {
  (void)cache;
  return int2e_one(out, dims, shls, atm, natm, bas, nbas, env, opt, 1);
}

int int2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
               double *env, CINTOpt *opt, double *cache) {
  (void)cache;
  return int2e_one(out, dims, shls, atm, natm, bas, nbas, env, opt, 0);
}

void int2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env) {
  if (!opt) return;
  *opt = nullptr;
  const long long nenv = env_extent(atm, natm, bas, nbas);
  if (check_common(atm, natm, bas, nbas, env, nenv)) return;
  LrbCintOpt *o = new LrbCintOpt();
  if (o->mol.upload(nullptr, atm, natm, bas, nbas, env, nenv) ||
      cudaStreamSynchronize(nullptr) != cudaSuccess) {
    o->mol.release(nullptr);
    delete o;
    return;
  }
  o->h_atm = atm; o->h_bas = bas; o->h_env = env;
  *opt = o;
}

void CINTdel_optimizer(CINTOpt **opt) {
  if (!opt || !*opt) return;
  (*opt)->mol.release(nullptr);
  cudaStreamSynchronize(nullptr);
  delete *opt;
  *opt = nullptr;
}

// ------------------------------------------------------------ p2c ABI
void free_c(double *ptr, size_t len) {
  (void)len;
  std::free(ptr);
}

double *int2e_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l,
                int coord) {
  const int natm = (int)(atm_l / 6);
  int nbas = (int)(bas_l / 8);
  if (coord != 0 && coord != 1) return set_error("coord must be 0 or 1"), nullptr;
  if (check_common(atm_p, natm, bas_p, nbas, env_p, (long long)env_l)) return nullptr;
  // generally contracted shells: the tensor of the segmented sub-shells is
  // the same tensor (same AO order)
  GcExpanded x;
  if (gc_expand(bas_p, nbas, env_p, (long long)env_l, x)) return nullptr;
  const int gc_screen = x.any ? 1 : 0;
  if (x.any) {
    bas_p = x.bas.data();
    nbas = (int)(x.bas.size() / 8);
    env_p = x.env.data();
    env_l = x.env.size();
  }
  std::vector<int> aooff(nbas + 1, 0), dim(nbas);
  for (int s = 0; s < nbas; ++s) {
    dim[s] = shell_dim(coord, bas_p, s);
    aooff[s + 1] = aooff[s] + dim[s];
  }
  const long long n = aooff[nbas];
  const long long n4 = n * n * n * n;
  // canonical quartets i>=j, k>=l, (ij)>=(kl)
  std::vector<int> quart;
  for (int i = 0; i < nbas; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= i; ++k)
        for (int l = 0; l <= (k == i ? j : k); ++l) {
          quart.push_back(i); quart.push_back(j); quart.push_back(k); quart.push_back(l);
        }
  const long long nq = (long long)quart.size() / 4;
  std::vector<long long> boff(nq + 1, 0);
  for (long long q = 0; q < nq; ++q)
    boff[q + 1] = boff[q] + (long long)dim[quart[4 * q]] * dim[quart[4 * q + 1]] *
                                dim[quart[4 * q + 2]] * dim[quart[4 * q + 3]];
  double *R = (double *)std::malloc(sizeof(double) * (size_t)std::max(n4, 1LL));
  if (!R) return set_error("host allocation failed"), nullptr;
  cudaStream_t st = nullptr;
  DevMol m;
  int *d_q = nullptr, *d_ao = nullptr, *d_dim = nullptr;
  long long *d_boff = nullptr;
  double *d_blk = nullptr, *d_R = nullptr;
  int rc = m.upload(st, atm_p, natm, bas_p, nbas, env_p, (long long)env_l);
  auto al = [&](void **p, size_t b) {
    if (rc) return;
    if (cudaMallocAsync(p, std::max(b, (size_t)8), st) != cudaSuccess) {
      cudaGetLastError();
      rc = (set_error("device allocation failed"), LRB_ERR_ALLOC);
    }
  };
  al((void **)&d_q, sizeof(int) * quart.size());
  al((void **)&d_ao, sizeof(int) * aooff.size());
  al((void **)&d_dim, sizeof(int) * dim.size());
  al((void **)&d_boff, sizeof(long long) * boff.size());
  al((void **)&d_blk, sizeof(double) * (size_t)boff[nq]);
  al((void **)&d_R, sizeof(double) * (size_t)n4);
  if (!rc) {
    cudaMemcpyAsync(d_q, quart.data(), sizeof(int) * quart.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_ao, aooff.data(), sizeof(int) * aooff.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_dim, dim.data(), sizeof(int) * dim.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_boff, boff.data(), sizeof(long long) * boff.size(), cudaMemcpyHostToDevice, st);
    rc = eri_batch_device(engine(), d_blk, coord, d_q, nq, m.atm, natm, m.bas, nbas, m.env,
                          (long long)env_l, st, nullptr, nullptr, gc_screen);
  }
  if (!rc) {
    k_scatter8<<<(unsigned)nq, 128, 0, st>>>(d_blk, d_boff, d_q, d_ao, d_dim, (int)nq, n, d_R);
    if (cudaGetLastError() != cudaSuccess) rc = LRB_ERR_CUDA;
  }
  if (!rc && cudaMemcpyAsync(R, d_R, sizeof(double) * (size_t)n4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = LRB_ERR_CUDA;
  for (void *p : {(void *)d_q, (void *)d_ao, (void *)d_dim, (void *)d_boff, (void *)d_blk, (void *)d_R})
    if (p) cudaFreeAsync(p, st);
  m.release(st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = LRB_ERR_CUDA;
  if (rc) {
    std::free(R);
    return nullptr;
  }
  return R;
}

// ------------------------------------------------------------ molecule / Fock / SCF
struct LrbMol {
  MolCtx ctx;
};

LRB_API int lrb_mol_create(LrbMol **out, const int *atm, int natm, const int *bas, int nbas,
                           const double *env, long long nenv) {
  if (!out) return set_error("NULL handle pointer"), LRB_ERR_INPUT;
  *out = nullptr;
  int rc = check_common(atm, natm, bas, nbas, env, nenv);
  if (rc) return rc;
  LrbMol *m = new LrbMol();
  rc = mol_create(m->ctx, atm, natm, bas, nbas, env, nenv, nullptr);
  if (rc) {
    mol_destroy(m->ctx, nullptr);
    delete m;
    return rc;
  }
  *out = m;
  return LRB_OK;
}

LRB_API void lrb_mol_destroy(LrbMol *m) {
  if (!m) return;
  mol_destroy(m->ctx, nullptr);
  delete m;
}

LRB_API int lrb_mol_nao(const LrbMol *m) { return m ? m->ctx.nao : -1; }

LRB_API int lrb_fock_G_device(LrbMol *m, const double *P, double *G, double tau, void *stream) {
  if (!m || !P || !G) return set_error("NULL argument"), LRB_ERR_INPUT;
  return fock_build(m->ctx, P, G, tau, (cudaStream_t)stream, nullptr);
}

LRB_API int lrb_fock_G(LrbMol *m, const double *P, double *G, double tau, long long *quartets) {
  if (!m || !P || !G) return set_error("NULL argument"), LRB_ERR_INPUT;
  const size_t nn = (size_t)m->ctx.nao * m->ctx.nao;
  cudaStream_t st = nullptr;
  double *dP = nullptr, *dG = nullptr;
  if (alloc_pair(st, nn, &dP, nn, &dG)) return LRB_ERR_ALLOC;
  cudaMemcpyAsync(dP, P, nn * 8, cudaMemcpyHostToDevice, st);
  FockStats fs;
  int rc = fock_build(m->ctx, dP, dG, tau, st, &fs);
  if (!rc) cudaMemcpyAsync(G, dG, nn * 8, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dP, st);
  cudaFreeAsync(dG, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  if (quartets) *quartets = fs.quartets;
  return rc;
}

LRB_API int lrb_fock_G_prec(LrbMol *m, const double *P, double *G, double tau, int prec,
                            double tau32, long long *quartets, long long *fp32_quartets) {
  if (!m || !P || !G) return set_error("NULL argument"), LRB_ERR_INPUT;
  if (prec < 0 || prec > 2) return set_error("prec must be 0, 1 or 2"), LRB_ERR_INPUT;
  const size_t nn = (size_t)m->ctx.nao * m->ctx.nao;
  cudaStream_t st = nullptr;
  double *dP = nullptr, *dG = nullptr;
  if (alloc_pair(st, nn, &dP, nn, &dG)) return LRB_ERR_ALLOC;
  cudaMemcpyAsync(dP, P, nn * 8, cudaMemcpyHostToDevice, st);
  FockStats fs;
  int rc = fock_build(m->ctx, dP, dG, tau, st, &fs, prec, tau32, false);
  if (!rc) cudaMemcpyAsync(G, dG, nn * 8, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dP, st);
  cudaFreeAsync(dG, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  if (quartets) *quartets = fs.quartets;
  if (fp32_quartets) *fp32_quartets = fs.fp32_quartets;
  return rc;
}

LRB_API int lrb_fock_G_part_device(LrbMol *m, const double *P, double *G, double tau, int rank,
                                   int nranks, long long *quartets, void *stream) {
  if (!m || !P || !G) return set_error("NULL argument"), LRB_ERR_INPUT;
  FockStats fs;
  const int rc = fock_build(m->ctx, P, G, tau, (cudaStream_t)stream, &fs, 0, 0.0, false, rank,
                            nranks);
  if (quartets) *quartets = fs.quartets;
  return rc;
}

LRB_API int lrb_fock_G_part(LrbMol *m, const double *P, double *G, double tau, int rank,
                            int nranks, long long *quartets) {
  if (!m || !P || !G) return set_error("NULL argument"), LRB_ERR_INPUT;
  const size_t nn = (size_t)m->ctx.nao * m->ctx.nao;
  cudaStream_t st = nullptr;
  double *dP = nullptr, *dG = nullptr;
  if (alloc_pair(st, nn, &dP, nn, &dG)) return LRB_ERR_ALLOC;
  cudaMemcpyAsync(dP, P, nn * 8, cudaMemcpyHostToDevice, st);
  int rc = lrb_fock_G_part_device(m, dP, dG, tau, rank, nranks, quartets, st);
  if (!rc) cudaMemcpyAsync(G, dG, nn * 8, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dP, st);
  cudaFreeAsync(dG, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  return rc;
}

LRB_API int lrb_scf(LrbMol *m, long long nelec, const LrbScfOptions *opt, LrbScfResult *res,
                    double *P_out, const double *P0) {
  if (!m) return set_error("NULL molecule"), LRB_ERR_INPUT;
  ScfOptions o;
  if (opt) {
    o.max_iter = opt->max_iter; o.conv = opt->conv; o.guess = opt->guess; o.diis = opt->diis;
    o.tau = opt->tau; o.mixed = opt->mixed; o.fp32_until = opt->fp32_until;
    o.tau32 = opt->tau32; o.rebuild_every = opt->rebuild_every > 0 ? opt->rebuild_every : 6;
    o.tau_fp32 = opt->tau_fp32;
    o.tau_prim = opt->tau_prim;
  }
  ScfResult r;
  // the SCF's Fock builds screen primitive quartets at tau_prim (when > 0)
  const double keep_prim = m->ctx.tau_prim;
  if (o.tau_prim > 0.0) m->ctx.tau_prim = o.tau_prim;
  const int rc = scf_run(m->ctx, (size_t)nelec, o, &r, P_out, P0, nullptr);
  m->ctx.tau_prim = keep_prim;
  if (res) {
    res->energy = r.energy; res->e_nuc = r.e_nuc; res->delta = r.delta; res->fock_ms = r.fock_ms;
    res->wall_ms = r.wall_ms; res->iterations = r.iterations; res->converged = r.converged;
    res->quartets = r.quartets; res->fp32_quartets = r.fp32_quartets;
  }
  return rc;
}

LRB_API int lrb_mol_set_tau_prim(LrbMol *m, double tau_prim) {
  if (!m || !(tau_prim >= 0.0)) return set_error("need a molecule and tau_prim >= 0"), LRB_ERR_INPUT;
  m->ctx.tau_prim = tau_prim;
  return LRB_OK;
}

LRB_API int lrb_energy(LrbMol *m, const double *P, double tau, double *E) {
  if (!m || !P || !E) return set_error("NULL argument"), LRB_ERR_INPUT;
  return energy_at(m->ctx, P, tau, E, nullptr);
}

LRB_API int lrb_int1e(LrbMol *m, int typec, int coord, double *out) {
  if (!m || !out) return set_error("NULL argument"), LRB_ERR_INPUT;
  if (typec < 0 || typec > 2 || coord < 0 || coord > 1) return set_error("bad typec/coord"), LRB_ERR_INPUT;
  MolCtx &c = m->ctx;
  int n = 0;
  for (int s = 0; s < c.nbas; ++s) n += shell_dim(coord, c.h_bas.data(), s);
  cudaStream_t st = nullptr;
  double *d = nullptr;
  if (cudaMallocAsync((void **)&d, sizeof(double) * (size_t)n * n, st) != cudaSuccess)
    return set_error("allocation failed"), LRB_ERR_ALLOC;
  double c2s[5 * 9 * 15];
  fill_c2s(c2s);
  int rc = int1e_device(typec, coord, c.atm, c.natm, c.bas, c.nbas, c.env, c.h_bas.data(), d, st, c2s);
  if (!rc) cudaMemcpyAsync(out, d, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  return rc;
}

// ---- p2c.rs shapes: inputs as (pointer, length), results malloc'd or in-band
static LrbMol *mol_from_p2c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                            size_t env_l) {
  LrbMol *m = nullptr;
  if (lrb_mol_create(&m, atm_p, (int)(atm_l / 6), bas_p, (int)(bas_l / 8), env_p, (long long)env_l))
    return nullptr;
  return m;
}

double *int1e_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l,
                int coord, int typec) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return nullptr;
  int n = 0;
  for (int s = 0; s < (int)(bas_l / 8); ++s) n += shell_dim(coord, bas_p, s);
  double *out = (double *)std::malloc(sizeof(double) * (size_t)n * n);
  if (!out || lrb_int1e(m, typec, coord, out)) {
    std::free(out);
    out = nullptr;
  }
  lrb_mol_destroy(m);
  return out;
}

double *density_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l,
                  size_t nelec, int imax, double conv) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return nullptr;
  const size_t nn = (size_t)m->ctx.nao * m->ctx.nao;
  double *P = (double *)std::malloc(sizeof(double) * nn);
  LrbScfOptions o{imax, conv, 0, 0, 0.0, 0, 0.0, 0.0, 6, 0.0, 0.0};
  if (!P || lrb_scf(m, (long long)nelec, &o, nullptr, P, nullptr)) {
    std::free(P);
    P = nullptr;
  }
  lrb_mol_destroy(m);
  return P;
}

double energy_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l,
                double *P_p, size_t P_l) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return NAN;
  double E = NAN;
  if ((size_t)m->ctx.nao * m->ctx.nao != P_l || lrb_energy(m, P_p, 0.0, &E)) E = NAN;
  lrb_mol_destroy(m);
  return E;
}

double scf_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l,
             size_t nelec, int imax, double conv) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return NAN;
  LrbScfOptions o{imax, conv, 0, 0, 0.0, 0, 0.0, 0.0, 6, 0.0, 0.0};
  LrbScfResult r;
  const int rc = lrb_scf(m, (long long)nelec, &o, &r, nullptr, nullptr);
  lrb_mol_destroy(m);
  return rc ? NAN : r.energy;
}

// ---- gradients with respect to env[s1:s2] (src/utils.rs:152-175 split)
// The reference's split: s1 = min PTR_EXP; s2 updated to PTR_COEFF + NPRIM
// whenever a shell's PTR_COEFF exceeds the current s2 (kept as written).
static void env_split(const int *bas, int nbas, int &s1, int &s2) {
  s1 = -1;
  s2 = -1;
  for (int s = 0; s < nbas; ++s) {
    const int ngto = bas[8 * s + 2], ex = bas[8 * s + 5], co = bas[8 * s + 6];
    if (s1 == -1 || s1 > ex) s1 = ex;
    if (s2 == -1) s2 = co + ngto;
    else if (s2 < co) s2 = co + ngto;
  }
}

LRB_API int lrb_grad_len(const LrbMol *m) {
  if (!m) return -1;
  int s1, s2;
  env_split(m->ctx.h_bas.data(), m->ctx.nbas, s1, s2);
  return s2 - s1;
}

LRB_API int lrb_grad(LrbMol *m, const double *P, double cH, double cR, double cS, double tau,
                     double *out) {
  if (!m || !P || !out) return set_error("NULL argument"), LRB_ERR_INPUT;
  MolCtx &c = m->ctx;
  int s1, s2;
  env_split(c.h_bas.data(), c.nbas, s1, s2);
  const size_t glen = (size_t)(c.nenv - s1), nn = (size_t)c.nao * c.nao;
  cudaStream_t st = nullptr;
  double *dP = nullptr, *dg = nullptr;
  if (alloc_pair(st, nn, &dP, glen, &dg)) return LRB_ERR_ALLOC;
  cudaMemcpyAsync(dP, P, nn * 8, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dg, 0, glen * 8, st);
  int rc = grad_run(c, dP, cH, cR, cS, tau, dg, s1, st);
  if (!rc) cudaMemcpyAsync(out, dg, sizeof(double) * (size_t)(s2 - s1), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dP, st);
  cudaFreeAsync(dg, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  return rc;
}

LRB_API int lrb_grad_nuc(LrbMol *m, const double *P, double tau, double *out) {
  if (!m || !P || !out) return set_error("NULL argument"), LRB_ERR_INPUT;
  MolCtx &c = m->ctx;
  const size_t nn = (size_t)c.nao * c.nao, ng = 3 * (size_t)c.natm;
  cudaStream_t st = nullptr;
  double *dP = nullptr, *dg = nullptr;
  if (alloc_pair(st, nn, &dP, ng, &dg)) return LRB_ERR_ALLOC;
  cudaMemcpyAsync(dP, P, nn * 8, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dg, 0, ng * 8, st);
  int rc = grad_nuc_run(c, dP, tau, dg, st);
  if (!rc) cudaMemcpyAsync(out, dg, ng * 8, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dP, st);
  cudaFreeAsync(dg, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  return rc;
}

LRB_API int lrb_int1e_jacobian(LrbMol *m, int typec, double *out) {
  if (!m || !out) return set_error("NULL argument"), LRB_ERR_INPUT;
  if (typec < 0 || typec > 2) return set_error("typec must be 0, 1 or 2"), LRB_ERR_INPUT;
  MolCtx &c = m->ctx;
  const size_t len = (size_t)c.nao * c.nao * (size_t)c.nenv;
  cudaStream_t st = nullptr;
  double *d = nullptr;
  if (cudaMallocAsync((void **)&d, sizeof(double) * std::max<size_t>(len, 1), st) != cudaSuccess)
    return set_error("allocation failed"), LRB_ERR_ALLOC;
  int rc = d1e_env_run(c, typec, d, st);
  if (!rc) cudaMemcpyAsync(out, d, sizeof(double) * len, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  return rc;
}

static double *grad_p2c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                        size_t env_l, double *P_p, size_t P_l, double cH, double cR, double cS) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return nullptr;
  double *out = nullptr;
  const int len = lrb_grad_len(m);
  if ((size_t)m->ctx.nao * m->ctx.nao == P_l && len > 0) {
    out = (double *)std::malloc(sizeof(double) * len);
    if (out && lrb_grad(m, P_p, cH, cR, cS, 0.0, out)) {
      std::free(out);
      out = nullptr;
    }
  } else {
    set_error("density size does not match the basis");
  }
  lrb_mol_destroy(m);
  return out;
}

// src/p2c.rs:131 dS_u: overlap Jacobian with respect to env[s1:s2], element
// (nu * n + mu) * (s2 - s1) + l (src/dscf.rs:96-151); n*n*(s2-s1) doubles.
double *dS_u(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p, size_t env_l) {
  LrbMol *m = mol_from_p2c(atm_p, atm_l, bas_p, bas_l, env_p, env_l);
  if (!m) return nullptr;
  int s1, s2;
  env_split(m->ctx.h_bas.data(), m->ctx.nbas, s1, s2);
  const size_t len = (size_t)m->ctx.nao * m->ctx.nao * (size_t)(s2 - s1);
  double *out = (double *)std::malloc(sizeof(double) * std::max<size_t>(len, 1));
  double *d = nullptr;
  cudaStream_t st = nullptr;
  int rc = out ? LRB_OK : (set_error("allocation failed"), LRB_ERR_ALLOC);
  if (!rc && cudaMallocAsync((void **)&d, sizeof(double) * std::max<size_t>(len, 1), st) != cudaSuccess)
    rc = (set_error("allocation failed"), LRB_ERR_ALLOC);
  if (!rc) rc = dS_u_run(m->ctx, s1, s2 - s1, d, st);
  if (!rc && cudaMemcpyAsync(out, d, sizeof(double) * len, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = (set_error("copy failed"), LRB_ERR_CUDA);
  if (d) cudaFreeAsync(d, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = (set_error("CUDA error"), LRB_ERR_CUDA);
  lrb_mol_destroy(m);
  if (rc) {
    std::free(out);
    return nullptr;
  }
  return out;
}

// src/p2c.rs:240 grad_c = dHcore + dR (src/dscf.rs:547-557)
double *grad_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P, size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 1.0, 1.0, 0.0);
}
// src/p2c.rs:267 dS_c = sum (PFP) dS (src/dscf.rs:354-368)
double *dS_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P, size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 0.0, 0.0, 1.0);
}
// src/p2c.rs:294 dHcore_c (src/dscf.rs:320-336)
double *dHcore_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P, size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 1.0, 0.0, 0.0);
}
// src/p2c.rs:321 dR_c (src/dscf.rs:370-524)
double *dR_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P, size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 0.0, 1.0, 0.0);
}
// src/p2c.rs:348 danalytical_c = dH + dR - dS/2 (src/dscf.rs:526-537)
double *danalytical_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P,
                      size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 1.0, 1.0, -0.5);
}
// src/p2c.rs:376 denergy_c delegates to the same assembly (src/dscf.rs:559-565)
double *denergy_c(int *a, size_t al, int *b, size_t bl, double *e, size_t el, double *P,
                  size_t Pl) {
  return grad_p2c(a, al, b, bl, e, el, P, Pl, 1.0, 1.0, -0.5);
}

}  // extern "C"
