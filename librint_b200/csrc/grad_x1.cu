// Adjoint ERI kernels with the differentiated shell of momentum 1, environment modes (coefficient, exponent);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x1(GradEntry *t) {
  t[NGRADMODE * 18 + 0] = make_grad_entry<1, 0, 0, 0, 0>();
  t[NGRADMODE * 18 + 1] = make_grad_entry<1, 0, 0, 0, 2>();
  t[NGRADMODE * 19 + 0] = make_grad_entry<1, 0, 1, 0, 0>();
  t[NGRADMODE * 19 + 1] = make_grad_entry<1, 0, 1, 0, 2>();
  t[NGRADMODE * 20 + 0] = make_grad_entry<1, 0, 1, 1, 0>();
  t[NGRADMODE * 20 + 1] = make_grad_entry<1, 0, 1, 1, 2>();
  t[NGRADMODE * 21 + 0] = make_grad_entry<1, 0, 2, 0, 0>();
  t[NGRADMODE * 21 + 1] = make_grad_entry<1, 0, 2, 0, 2>();
  t[NGRADMODE * 22 + 0] = make_grad_entry<1, 0, 2, 1, 0>();
  t[NGRADMODE * 22 + 1] = make_grad_entry<1, 0, 2, 1, 2>();
  t[NGRADMODE * 23 + 0] = make_grad_entry<1, 0, 2, 2, 0>();
  t[NGRADMODE * 23 + 1] = make_grad_entry<1, 0, 2, 2, 2>();
  t[NGRADMODE * 24 + 0] = make_grad_entry<1, 1, 0, 0, 0>();
  t[NGRADMODE * 24 + 1] = make_grad_entry<1, 1, 0, 0, 2>();
  t[NGRADMODE * 25 + 0] = make_grad_entry<1, 1, 1, 0, 0>();
  t[NGRADMODE * 25 + 1] = make_grad_entry<1, 1, 1, 0, 2>();
  t[NGRADMODE * 26 + 0] = make_grad_entry<1, 1, 1, 1, 0>();
  t[NGRADMODE * 26 + 1] = make_grad_entry<1, 1, 1, 1, 2>();
  t[NGRADMODE * 27 + 0] = make_grad_entry<1, 1, 2, 0, 0>();
  t[NGRADMODE * 27 + 1] = make_grad_entry<1, 1, 2, 0, 2>();
  t[NGRADMODE * 28 + 0] = make_grad_entry<1, 1, 2, 1, 0>();
  t[NGRADMODE * 28 + 1] = make_grad_entry<1, 1, 2, 1, 2>();
  t[NGRADMODE * 29 + 0] = make_grad_entry<1, 1, 2, 2, 0>();
  t[NGRADMODE * 29 + 1] = make_grad_entry<1, 1, 2, 2, 2>();
  t[NGRADMODE * 30 + 0] = make_grad_entry<1, 2, 0, 0, 0>();
  t[NGRADMODE * 30 + 1] = make_grad_entry<1, 2, 0, 0, 2>();
  t[NGRADMODE * 31 + 0] = make_grad_entry<1, 2, 1, 0, 0>();
  t[NGRADMODE * 31 + 1] = make_grad_entry<1, 2, 1, 0, 2>();
  t[NGRADMODE * 32 + 0] = make_grad_entry<1, 2, 1, 1, 0>();
  t[NGRADMODE * 32 + 1] = make_grad_entry<1, 2, 1, 1, 2>();
  t[NGRADMODE * 33 + 0] = make_grad_entry<1, 2, 2, 0, 0>();
  t[NGRADMODE * 33 + 1] = make_grad_entry<1, 2, 2, 0, 2>();
  t[NGRADMODE * 34 + 0] = make_grad_entry<1, 2, 2, 1, 0>();
  t[NGRADMODE * 34 + 1] = make_grad_entry<1, 2, 2, 1, 2>();
  t[NGRADMODE * 35 + 0] = make_grad_entry<1, 2, 2, 2, 0>();
  t[NGRADMODE * 35 + 1] = make_grad_entry<1, 2, 2, 2, 2>();
}

}  // namespace lrb
