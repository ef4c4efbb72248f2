// Batched ERIs with no device allocation (lrb_int2e_batch_device_noalloc).
//
// Who needs it: callers that may not allocate device memory at the moment
// they want integrals.  Examples are a host framework whose caching
// allocator has already reserved the GPU's free memory (a further
// cudaMalloc would fail, or would force the framework to release its
// cache), and latency-bound loops that cannot afford the device-wide
// synchronisation of cudaMalloc/cudaFree or the page mapping of a fresh
// pool allocation.  lrb_int2e_batch_device takes its scratch (quartet table,
// sort keys, CUB temporary storage, primitive pairs) from a grow-only pool;
// this entry point takes all of it from one file-scope device array instead.
//
// Rules for callers:
//  * The array is LRB_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU that loads
//    this library holds it until the process exits.
//  * A batch is rejected (LRB_ERR_INPUT, with the sizes in lrb_last_error())
//    when it has more than LRB_NOALLOC_MAX_QUARTETS quartets or when its
//    quartet tables plus primitive pairs do not fit; split such batches.
//  * All calls share the array and it keeps the previous call's contents.
//    The only state that must start at zero (the per-class work counters,
//    the error flag and the primitive-pair counter) is cleared by every call
//    on its own stream; everything else is written before it is read.
//    Calls whose GPU work overlaps (different streams without ordering
//    between them, or different host threads) race on the array: order them.
//  * The first call on a device looks up the array's device address and
//    sets up the kernel table; make that first call before any stream
//    capture starts.  With CUDA's default lazy module loading the array
//    itself is only placed in device memory at that first call, so make the
//    first call (a warm-up call will do) before the framework reserves the
//    GPU's free memory, or load modules eagerly (CUDA_MODULE_LOADING=EAGER);
//    an out-of-memory failure of that first call says so.
//  * It synchronises `stream` three times while preparing the batch: after
//    counting the primitive pairs, after checking the molecule's indices,
//    and after reading back the block sizes and class boundaries.
//  * Kernel timing (lrb_profile_enable) and the launch counter
//    (lrb_launch_count) cover this entry point like the others.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "engine.h"
#include "eri_device.cuh"

namespace lrb {
namespace {

// The scratch.  Host code may not use this name as an address (on the host
// it is only a stand-in); the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LRB_NOALLOC_SCRATCH_BYTES];

struct NoallocDevice {
  char *base = nullptr;   // device address of g_noalloc_scratch
  Engine eng;             // its workspace arenas point into the scratch
};
constexpr int kMaxDevices = 64;
NoallocDevice g_noalloc[kMaxDevices];
std::mutex g_noalloc_mu;

inline size_t up256(size_t n) { return (n + 255) & ~size_t(255); }

// Sum over quartets of (bra + ket) primitive pairs; shells out of range are
// skipped here and reported by the batch driver.
__global__ void k_count_pairs(const int *__restrict__ shls, long long nq,
                              const int *__restrict__ bas, int nbas,
                              unsigned long long *__restrict__ total) {
  unsigned long long s = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    int k[4];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int sh = shls[4 * q + a];
      ok = ok && sh >= 0 && sh < nbas;
      k[a] = ok ? bas[8 * sh + 2] : 0;
    }
    if (ok) s += (unsigned long long)k[0] * k[1] + (unsigned long long)k[2] * k[3];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

int noalloc_setup(int dev, NoallocDevice *&nd) {
  if (dev < 0 || dev >= kMaxDevices) return set_error("device index out of range"), LRB_ERR_INPUT;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  nd = &g_noalloc[dev];
  if (nd->base) return LRB_OK;
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    char msg[320];
    if (e == cudaErrorMemoryAllocation)
      snprintf(msg, sizeof msg,
               "no-alloc scratch: the %llu-byte static array could not be placed in device "
               "memory (%s); make the first call before other code reserves the GPU's free "
               "memory, or set CUDA_MODULE_LOADING=EAGER so it is placed when the library loads",
               (unsigned long long)LRB_NOALLOC_SCRATCH_BYTES, cudaGetErrorString(e));
    else
      snprintf(msg, sizeof msg, "no-alloc scratch: cudaGetSymbolAddress failed (%s)",
               cudaGetErrorString(e));
    cudaGetLastError();
    return set_error(msg), LRB_ERR_CUDA;
  }
  nd->base = static_cast<char *>(p);
  for (Arena *a : {&nd->eng.ws.main, &nd->eng.ws.aux, &nd->eng.ws.pairs, &nd->eng.ws.extra}) {
    a->ptr = nullptr;
    a->size = 0;
    a->fixed = true;
  }
  return LRB_OK;
}

}  // namespace
}  // namespace lrb

using namespace lrb;

extern "C" LRB_API int lrb_int2e_batch_device_noalloc(double *out, int coord, const int *shls,
                                                      long long nq, const int *atm, int natm,
                                                      const int *bas, int nbas, const double *env,
                                                      long long nenv, void *stream) {
  if (nq == 0) return LRB_OK;
  if (!out || !shls || nq < 0 || !atm || !bas || !env || nbas <= 0)
    return set_error("bad output, quartet list or molecule"), LRB_ERR_INPUT;
  if (nq > LRB_NOALLOC_MAX_QUARTETS) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "no-alloc batch of %lld quartets exceeds the limit of %d; split the batch", nq,
             (int)LRB_NOALLOC_MAX_QUARTETS);
    return set_error(msg), LRB_ERR_INPUT;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error("no current device"), LRB_ERR_CUDA;
  NoallocDevice *nd = nullptr;
  int rc = noalloc_setup(dev, nd);
  if (rc) return rc;

  // Layout of the scratch for this call: [pair counter | quartet tables |
  // CUB temporary storage | primitive pairs].  The first two requests match
  // what the batch driver asks its workspace for.
  const size_t q = (size_t)nq;
  const size_t main_need = q * sizeof(QuartetJob) * 2 + q * (4 * sizeof(unsigned) + 4 * sizeof(int)) +
                           q * 2 * sizeof(long long) + q * 4 * sizeof(int) + (size_t)nbas * 24 +
                           4096 + (1 << 20);
  size_t t1 = 0, t2 = 0, t3 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, t1, (long long *)nullptr, (long long *)nullptr, (int)nq, st);
  cub::DeviceScan::ExclusiveSum(nullptr, t2, (int *)nullptr, (int *)nullptr, (int)(2 * nq), st);
  cub::DeviceRadixSort::SortPairs(nullptr, t3, (unsigned *)nullptr, (unsigned *)nullptr,
                                  (int *)nullptr, (int *)nullptr, (int)nq, 0, 32, st);
  const size_t aux_need = std::max(t1, std::max(t2, t3)) + 2 * sizeof(long long) + 2 * sizeof(int) + 64;
  const size_t o_main = 256, o_aux = o_main + up256(main_need), o_pairs = o_aux + up256(aux_need);
  const size_t cap = LRB_NOALLOC_SCRATCH_BYTES;
  if (o_pairs >= cap) {
    char msg[220];
    snprintf(msg, sizeof msg,
             "no-alloc batch: quartet tables need %zu bytes of the %zu-byte scratch; split the batch",
             o_pairs, cap);
    return set_error(msg), LRB_ERR_INPUT;
  }
  // primitive pairs of the batch (raw and sorted copies)
  unsigned long long *d_npp = reinterpret_cast<unsigned long long *>(nd->base);
  unsigned long long npp = 0;
  if (cudaMemsetAsync(d_npp, 0, sizeof(unsigned long long), st) != cudaSuccess)
    return set_error("no-alloc batch: memset failed"), LRB_ERR_CUDA;
  k_count_pairs<<<(unsigned)std::min<long long>((nq + 255) / 256, 1024), 256, 0, st>>>(
      shls, nq, bas, nbas, d_npp);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&npp, d_npp, sizeof npp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return set_error("no-alloc batch: counting primitive pairs failed"), LRB_ERR_CUDA;
  const size_t pairs_need = 2 * (size_t)std::max(npp, 1ull) * sizeof(PrimPair);
  if (pairs_need > cap - o_pairs) {
    char msg[260];
    snprintf(msg, sizeof msg,
             "no-alloc batch: %llu primitive pairs need %zu bytes but %zu of the %zu-byte "
             "scratch are left after the quartet tables; split the batch",
             npp, pairs_need, cap - o_pairs, cap);
    return set_error(msg), LRB_ERR_INPUT;
  }
  Workspace &w = nd->eng.ws;
  w.main.ptr = nd->base + o_main;
  w.main.size = o_aux - o_main;
  w.aux.ptr = nd->base + o_aux;
  w.aux.size = o_pairs - o_aux;
  w.pairs.ptr = nd->base + o_pairs;
  w.pairs.size = cap - o_pairs;
  // the shared engine's settings and counters cover this entry point too
  Engine &shared = engine();
  nd->eng.expcutoff = shared.expcutoff;
  nd->eng.profile = shared.profile;
  const long long launches0 = nd->eng.launches;
  rc = eri_batch_device(nd->eng, out, coord, shls, nq, atm, natm, bas, nbas, env, nenv, st, nullptr);
  shared.launches += nd->eng.launches - launches0 + 1;   // + k_count_pairs
  for (ProfRecord &r : nd->eng.prof) shared.prof.push_back(r);
  nd->eng.prof.clear();
  if (rc == LRB_ERR_ALLOC)
    set_error("no-alloc batch: the batch needs more scratch than this entry point has; split it");
  return rc;
}
