// Engine state shared by the kernels' host drivers: error reporting and a
// grow-only, stream-ordered device workspace (cudaMallocAsync), one per
// device.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "../../include/librint_b200.h"

namespace lrb {

constexpr int ERI_LMAX = 3;    // shells up to f (d: templated kernels, f: eri_gen.cu)
constexpr int ERI_KMAX = 31;   // primitives per shell (sort-key packing limit)

void set_error(const char *msg);

// Grow-only device arena; growth frees the old block on the same stream, so
// work already queued on that stream finishes before the memory is reused.
struct Arena {
  char *ptr = nullptr;
  size_t size = 0;
  bool fixed = false;   // caller-provided memory: never freed or grown
  char *get(cudaStream_t st, size_t need);
};

struct Workspace {
  Arena main, aux, pairs, extra;
  char *reserve(cudaStream_t st, size_t n) { return main.get(st, n); }
  void *reserve_aux(cudaStream_t st, size_t n) { return aux.get(st, n); }
  void *reserve_pairs(cudaStream_t st, size_t n) { return pairs.get(st, n); }
  void *reserve_extra(cudaStream_t st, size_t n) { return extra.get(st, n); }
};

// Carves 256-byte aligned sub-buffers out of one allocation.
struct Carver {
  char *p;
  explicit Carver(char *base) : p(base) {}
  template <class T>
  T *take(size_t n) {
    T *r = reinterpret_cast<T *>(p);
    p += (n * sizeof(T) + 255) & ~size_t(255);
    return r;
  }
};
inline size_t carve_size(size_t bytes) { return (bytes + 255) & ~size_t(255); }

// Per-kernel timing for measurement: CUDA events recorded around each ERI
// class kernel on its own stream while profiling is enabled.
struct ProfRecord {
  int cls;
  cudaEvent_t start, stop;
};

struct Engine {
  Workspace ws;
  double expcutoff = 60.0;   // reference default, src/g2e.rs:83-92
  bool profile = false;
  std::vector<ProfRecord> prof;
  long long launches = 0;    // kernels of this library launched so far
  // Fock-build class counts while profiling (index = Fock class id: class,
  // +55 for the FP32 kernels): shell quartets, and on the device the
  // primitive quartets that passed screening
  long long fock_quartets[128] = {};
  unsigned long long *fock_prim = nullptr;   // 128 device counters
  // host-buffer entry points: three non-blocking streams (copies in,
  // kernels, copies out) so that one chunk's copy in, the previous chunk's
  // kernels and the one before's copy out run at the same time; two device
  // slots for quartet lists and outputs (chunk c uses slot c % 2) that only
  // grow, and the events that hand a slot from one stream to the next
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_cmp[2] = {nullptr, nullptr},
              ev_out[2] = {nullptr, nullptr};
  Arena pipe_out[2], pipe_in[2], pipe_centers;
};
Engine &engine();          // for the current device

struct EriBatchStats {
  long long nq = 0, out_len = 0, prim_pairs = 0;
};

// centers_ready: shell centres already computed (and the molecule's indices
// checked) by eri_centers for this molecule; NULL computes them per call.
// gc_screen: bas slot 7 of a shell, when positive, points at the screening
// coefficients (largest |c| over the contractions of the generally contracted
// shell it was split from); set only for bas arrays built by gc_expand.
int eri_batch_device(Engine &eng, double *out, int coord, const int *d_shls, long long nq,
                     const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                     long long nenv, cudaStream_t st, EriBatchStats *stats,
                     const double *centers_ready = nullptr, int gc_screen = 0);

// Generally contracted shells (nctr > 1) as nctr consecutive segmented
// sub-shells with the same exponents (coefficient pointer advanced by
// c * nprim), so the AO numbering is unchanged.  env gains, per such shell,
// the largest |coefficient| of each primitive over its contractions (the
// reference's screening coefficient, src/optimizer.rs:661-687), referenced by
// the sub-shells' bas slot 7.  any == false: nothing to expand.
struct GcExpanded {
  bool any = false;
  std::vector<int> bas;      // 8 ints per sub-shell
  std::vector<double> env;   // the input env followed by the screening arrays
  std::vector<int> first;    // first sub-shell of each input shell (nbas + 1)
};
int gc_expand(const int *bas, int nbas, const double *env, long long nenv, GcExpanded &x);
// Shell centres (3 doubles per shell) with every atm/bas/env index checked;
// d_err is one device int; synchronises st to read it.
int eri_centers(const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                long long nenv, double *centers, int *d_err, cudaStream_t st);
long long eri_batch_out_len(int coord, const int *shls, long long nq, const int *bas);
// k_centers over nbas shells starting at d_bas (centres written from
// `centers`), queued on st without reading the error flag back: for shells
// whose indices the caller has checked on the host.
void eri_centers_async(const int *d_atm, int natm, const int *d_bas, int nbas, const double *d_env,
                       long long nenv, double *centers, int *d_err, cudaStream_t st);

}  // namespace lrb
