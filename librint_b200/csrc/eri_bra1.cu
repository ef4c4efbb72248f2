// Kernels of the classes with bra (ps| -- generated list, one TU per bra.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "eri_classes.cuh"

namespace lrb {

cudaError_t eri_register_bra1(ClassEntry *t, const double *c2s_host) {
  const cudaError_t e = cudaMemcpyToSymbol(c_c2s, c2s_host, sizeof(c_c2s));
  if (e != cudaSuccess || !t) return e;
  t[class_id(1, 0, 0, 0)] = make_entry<1, 0, 0, 0>();
  t[class_id(1, 0, 1, 0)] = make_entry<1, 0, 1, 0>();
  return cudaSuccess;
}

}  // namespace lrb
