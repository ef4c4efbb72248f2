// Adjoint ERI kernels with the differentiated shell of momentum 2, environment modes (coefficient, exponent);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x2(GradEntry *t) {
  t[NGRADMODE * 36 + 0] = make_grad_entry<2, 0, 0, 0, 0>();
  t[NGRADMODE * 36 + 1] = make_grad_entry<2, 0, 0, 0, 2>();
  t[NGRADMODE * 37 + 0] = make_grad_entry<2, 0, 1, 0, 0>();
  t[NGRADMODE * 37 + 1] = make_grad_entry<2, 0, 1, 0, 2>();
  t[NGRADMODE * 38 + 0] = make_grad_entry<2, 0, 1, 1, 0>();
  t[NGRADMODE * 38 + 1] = make_grad_entry<2, 0, 1, 1, 2>();
  t[NGRADMODE * 39 + 0] = make_grad_entry<2, 0, 2, 0, 0>();
  t[NGRADMODE * 39 + 1] = make_grad_entry<2, 0, 2, 0, 2>();
  t[NGRADMODE * 40 + 0] = make_grad_entry<2, 0, 2, 1, 0>();
  t[NGRADMODE * 40 + 1] = make_grad_entry<2, 0, 2, 1, 2>();
  t[NGRADMODE * 41 + 0] = make_grad_entry<2, 0, 2, 2, 0>();
  t[NGRADMODE * 41 + 1] = make_grad_entry<2, 0, 2, 2, 2>();
  t[NGRADMODE * 42 + 0] = make_grad_entry<2, 1, 0, 0, 0>();
  t[NGRADMODE * 42 + 1] = make_grad_entry<2, 1, 0, 0, 2>();
  t[NGRADMODE * 43 + 0] = make_grad_entry<2, 1, 1, 0, 0>();
  t[NGRADMODE * 43 + 1] = make_grad_entry<2, 1, 1, 0, 2>();
  t[NGRADMODE * 44 + 0] = make_grad_entry<2, 1, 1, 1, 0>();
  t[NGRADMODE * 44 + 1] = make_grad_entry<2, 1, 1, 1, 2>();
  t[NGRADMODE * 45 + 0] = make_grad_entry<2, 1, 2, 0, 0>();
  t[NGRADMODE * 45 + 1] = make_grad_entry<2, 1, 2, 0, 2>();
  t[NGRADMODE * 46 + 0] = make_grad_entry<2, 1, 2, 1, 0>();
  t[NGRADMODE * 46 + 1] = make_grad_entry<2, 1, 2, 1, 2>();
  t[NGRADMODE * 47 + 0] = make_grad_entry<2, 1, 2, 2, 0>();
  t[NGRADMODE * 47 + 1] = make_grad_entry<2, 1, 2, 2, 2>();
  t[NGRADMODE * 48 + 0] = make_grad_entry<2, 2, 0, 0, 0>();
  t[NGRADMODE * 48 + 1] = make_grad_entry<2, 2, 0, 0, 2>();
  t[NGRADMODE * 49 + 0] = make_grad_entry<2, 2, 1, 0, 0>();
  t[NGRADMODE * 49 + 1] = make_grad_entry<2, 2, 1, 0, 2>();
  t[NGRADMODE * 50 + 0] = make_grad_entry<2, 2, 1, 1, 0>();
  t[NGRADMODE * 50 + 1] = make_grad_entry<2, 2, 1, 1, 2>();
  t[NGRADMODE * 51 + 0] = make_grad_entry<2, 2, 2, 0, 0>();
  t[NGRADMODE * 51 + 1] = make_grad_entry<2, 2, 2, 0, 2>();
  t[NGRADMODE * 52 + 0] = make_grad_entry<2, 2, 2, 1, 0>();
  t[NGRADMODE * 52 + 1] = make_grad_entry<2, 2, 2, 1, 2>();
  t[NGRADMODE * 53 + 0] = make_grad_entry<2, 2, 2, 2, 0>();
  t[NGRADMODE * 53 + 1] = make_grad_entry<2, 2, 2, 2, 2>();
}

}  // namespace lrb
