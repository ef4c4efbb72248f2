// Class table of the ERI kernels: ids, dispatch entries and the per-bra
// registration functions (one translation unit each, eri_bra<P>.cu, so the
// kernels compile in parallel).
#pragma once
#include "engine.h"
#include "eri_kernel.cuh"

namespace lrb {

// Canonical classes for l <= ERI_LMAX, id = P(P+1)/2 + Q with pair index
// P = li(li+1)/2 + lj of the bra (li >= lj) and Q of the ket, P >= Q.
__host__ __device__ inline int pair_index(int a, int b) { return a * (a + 1) / 2 + b; }
__host__ __device__ inline int class_id(int li, int lj, int lk, int ll) {
  const int P = pair_index(li, lj), Q = pair_index(lk, ll);
  return P * (P + 1) / 2 + Q;
}
constexpr int NPAIRCLS = (ERI_LMAX + 1) * (ERI_LMAX + 2) / 2;
constexpr int NCLASS = NPAIRCLS * (NPAIRCLS + 1) / 2;   // 55 for l <= 3
constexpr int NCLASS_TPL = 21;   // l <= 2: the templated kernels; ids 21.. carry an f shell

using EriKernelFn = void (*)(EriParams, FockParams, const double *, int *);

// Classes with an f shell run k_eri_gen (eri_gen.cu), one quartet per CTA.
constexpr int GEN_THREADS = 128;
struct GenClass {
  int li, lj, lk, ll, nr;
  int ib, kb;              // bra base is i (else j); ket base is k (else l)
  int la, lb, lc, ld;      // base / partner momenta of bra and ket
  int ni, nj, nk, nl;      // cartesian counts
  int gsz;                 // (la+1)(lb+1)(lc+1)(ld+1)
};
using GenKernelFn = void (*)(EriParams, FockParams, GenClass, const double *, int *);
GenClass gen_class(int li, int lj, int lk, int ll);
GenKernelFn gen_kernel(int mode);                 // 0 output, 1 Fock (FP64)
size_t gen_smem_bytes(const GenClass &g, int mode);
cudaError_t eri_register_gen(const double *c2s_host);   // per device

struct ClassEntry {
  EriKernelFn fn[3];     // output (FP64), Fock digestion FP64, Fock digestion FP32
  size_t smem[3];
  EriKernelFn lp[2];     // Fock lane-per-primitive kernels (FP64, FP32) or NULL
  size_t lp_smem[2];
  int slots, nr;
  int gen;               // 1: k_eri_gen with `g` (fn unused)
  GenClass g;
};

template <int LI, int LJ, int LK, int LL>
ClassEntry make_entry() {
  using C = EriClass<LI, LJ, LK, LL, true>;
  ClassEntry e;
  e.fn[0] = k_eri<LI, LJ, LK, LL, 0>;
  e.fn[1] = k_eri<LI, LJ, LK, LL, 1>;
  e.fn[2] = k_eri<LI, LJ, LK, LL, 1, float>;
  e.smem[0] = EriLayout<C, 0>::SMEM;
  e.smem[1] = EriLayout<C, 1>::SMEM;
  e.smem[2] = EriLayout<C, 1, float>::SMEM;
  e.slots = C::SLOTS;
  e.nr = C::NR;
  e.gen = 0;
  e.lp[0] = e.lp[1] = nullptr;
  e.lp_smem[0] = e.lp_smem[1] = 0;
  if constexpr (lp_passes<LI, LJ, LK, LL, double>() > 0) {
    e.lp[0] = k_fock_lp<LI, LJ, LK, LL, double>;
    e.lp_smem[0] = LpLayout<LI, LJ, LK, LL, double>::SMEM;
  }
  if constexpr (lp_passes<LI, LJ, LK, LL, float>() > 0) {
    e.lp[1] = k_fock_lp<LI, LJ, LK, LL, float>;
    e.lp_smem[1] = LpLayout<LI, LJ, LK, LL, float>::SMEM;
  }
  return e;
}

// Class table.  The kernel pointers and shared-memory sizes are host data,
// filled once per process; the cart->sph constants of every translation unit
// and the large-shared-memory attribute of every kernel belong to a device
// and are set up once for each device the process uses.  Returns NULL (with
// the error set) when that per-device set-up fails.
const ClassEntry *class_table();
void fill_c2s(double *c);

// Each registration uploads its unit's cart->sph constants to the current
// device and, when t is not NULL, fills its classes' table entries.
cudaError_t eri_register_bra0(ClassEntry *t, const double *c2s_host);   // (ss|
cudaError_t eri_register_bra1(ClassEntry *t, const double *c2s_host);   // (ps|
cudaError_t eri_register_bra2(ClassEntry *t, const double *c2s_host);   // (pp|
cudaError_t eri_register_bra3(ClassEntry *t, const double *c2s_host);   // (ds|
cudaError_t eri_register_bra4(ClassEntry *t, const double *c2s_host);   // (dp|
cudaError_t eri_register_bra5(ClassEntry *t, const double *c2s_host);   // (dd|

}  // namespace lrb
