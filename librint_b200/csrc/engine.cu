#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"

namespace lrb {

static thread_local std::string g_err;

void set_error(const char *msg) { g_err = msg ? msg : ""; }
const char *last_error() { return g_err.c_str(); }

char *Arena::get(cudaStream_t st, size_t need) {
  if (need <= size) return ptr;
  if (fixed) return nullptr;
  if (ptr) cudaFreeAsync(ptr, st);
  size_t sz = need + need / 4 + (1 << 20);
  void *p = nullptr;
  if (cudaMallocAsync(&p, sz, st) != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    size = 0;
    return nullptr;
  }
  ptr = static_cast<char *>(p);
  size = sz;
  return ptr;
}

Engine &engine() {
  static std::mutex mu;
  static std::vector<Engine *> per_dev;   // indexed by device; engines live until exit
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if ((size_t)dev >= per_dev.size()) per_dev.resize((size_t)dev + 1, nullptr);
  if (!per_dev[dev]) {
    // keep freed stream-ordered memory in the device's default pool instead
    // of returning it to the driver at every synchronisation, so repeated
    // cudaMallocAsync of the same sizes does not remap pages
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    per_dev[dev] = new Engine();
  }
  return *per_dev[dev];
}

int gc_expand(const int *bas, int nbas, const double *env, long long nenv, GcExpanded &x) {
  x = GcExpanded();
  x.first.assign(nbas + 1, 0);
  for (int s = 0; s < nbas; ++s) {
    const int *b = bas + 8 * s;
    if (b[3] < 1 || b[2] < 1 || b[5] < 0 || b[6] < 0 || (long long)b[5] + b[2] > nenv ||
        (long long)b[6] + (long long)b[2] * b[3] > nenv)
      return set_error("bas entry out of range (nprim, nctr or env pointers)"), LRB_ERR_INPUT;
    x.first[s + 1] = x.first[s] + b[3];
    x.any = x.any || b[3] > 1;
  }
  if (!x.any) return LRB_OK;
  x.env.assign(env, env + nenv);
  x.bas.reserve(8 * (size_t)x.first[nbas]);
  for (int s = 0; s < nbas; ++s) {
    const int *b = bas + 8 * s;
    const int nprim = b[2], nctr = b[3];
    int scr = 0;
    if (nctr > 1) {
      scr = (int)x.env.size();
      for (int p = 0; p < nprim; ++p) {
        double m = 0.0;
        for (int c = 0; c < nctr; ++c) m = std::max(m, std::fabs(env[b[6] + c * nprim + p]));
        x.env.push_back(m);
      }
    }
    for (int c = 0; c < nctr; ++c) {
      const int sub[8] = {b[0], b[1], nprim, 1, b[4], b[5], b[6] + c * nprim, scr};
      x.bas.insert(x.bas.end(), sub, sub + 8);
    }
  }
  return LRB_OK;
}

// FP64 FMA throughput probe: 8 independent chains per thread keep the FP64
// pipe busy without memory traffic; the result is written so the work stays.
__global__ void k_fp64_probe(double *sink, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(x[k]) : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 12345.678) sink[0] = s;
}

}  // namespace lrb

using namespace lrb;

extern "C" {

LRB_API const char *lrb_last_error(void) { return lrb::last_error(); }

LRB_API void lrb_profile_enable(int on) {
  Engine &e = engine();
  e.profile = on != 0;
}

// Milliseconds per ERI class kernel accumulated since the last read, into
// ms[0..n); returns the number of records harvested (waits for them).
LRB_API int lrb_profile_read(double *ms, int n) {
  Engine &e = engine();
  for (int i = 0; i < n; ++i) ms[i] = 0.0;
  int cnt = 0;
  for (ProfRecord &r : e.prof) {
    cudaEventSynchronize(r.stop);
    float t = 0.f;
    cudaEventElapsedTime(&t, r.start, r.stop);
    if (r.cls >= 0 && r.cls < n) ms[r.cls] += t;
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
    ++cnt;
  }
  e.prof.clear();
  return cnt;
}

LRB_API long long lrb_launch_count(void) { return engine().launches; }

// Per Fock class (id = canonical class, +55 for the FP32 kernels) the shell
// quartets and the screened primitive quartets of the Fock builds run while
// profiling was enabled, since the last read; clears them.
LRB_API int lrb_fock_class_counts(long long *quartets, long long *prim_quartets, int n) {
  Engine &e = engine();
  unsigned long long h[128] = {};
  if (e.fock_prim) {
    if (cudaMemcpy(h, e.fock_prim, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(e.fock_prim, 0, sizeof h) != cudaSuccess)
      return set_error("fock class counts: copy failed"), LRB_ERR_CUDA;
  }
  for (int i = 0; i < n; ++i) {
    quartets[i] = i < 128 ? e.fock_quartets[i] : 0;
    prim_quartets[i] = i < 128 ? (long long)h[i] : 0;
  }
  for (long long &q : e.fock_quartets) q = 0;
  return LRB_OK;
}

// Measured FP64 FMA throughput of the current device in TFLOP/s (about
// `ms` milliseconds of work, timed with CUDA events).
LRB_API double lrb_fp64_peak_probe(int ms) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  double *sink = nullptr;
  if (cudaMalloc(&sink, 8) != cudaSuccess) return -1.0;
  const int threads = 256, blocks = nsm * 8;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int iters = 1 << 14, timed = iters;
  float t = 0.f;
  k_fp64_probe<<<blocks, threads>>>(sink, iters, 0.999999, 1e-9);   // warm-up
  for (int rep = 0; rep < 8; ++rep) {
    cudaEventRecord(a);
    k_fp64_probe<<<blocks, threads>>>(sink, iters, 0.999999, 1e-9);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&t, a, b);
    timed = iters;          // t belongs to this launch's iteration count
    if (t >= ms) break;
    iters *= 2;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (cudaGetLastError() != cudaSuccess || t <= 0.f) return -1.0;
  const double flops = 2.0 * 8.0 * (double)timed * threads * blocks;
  return flops / (t * 1e-3) / 1e12;
}

}  // extern "C"

