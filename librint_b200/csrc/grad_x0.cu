// Adjoint ERI kernels with the differentiated shell of momentum 0, environment modes (coefficient, exponent);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x0(GradEntry *t) {
  t[NGRADMODE * 0 + 0] = make_grad_entry<0, 0, 0, 0, 0>();
  t[NGRADMODE * 0 + 1] = make_grad_entry<0, 0, 0, 0, 2>();
  t[NGRADMODE * 1 + 0] = make_grad_entry<0, 0, 1, 0, 0>();
  t[NGRADMODE * 1 + 1] = make_grad_entry<0, 0, 1, 0, 2>();
  t[NGRADMODE * 2 + 0] = make_grad_entry<0, 0, 1, 1, 0>();
  t[NGRADMODE * 2 + 1] = make_grad_entry<0, 0, 1, 1, 2>();
  t[NGRADMODE * 3 + 0] = make_grad_entry<0, 0, 2, 0, 0>();
  t[NGRADMODE * 3 + 1] = make_grad_entry<0, 0, 2, 0, 2>();
  t[NGRADMODE * 4 + 0] = make_grad_entry<0, 0, 2, 1, 0>();
  t[NGRADMODE * 4 + 1] = make_grad_entry<0, 0, 2, 1, 2>();
  t[NGRADMODE * 5 + 0] = make_grad_entry<0, 0, 2, 2, 0>();
  t[NGRADMODE * 5 + 1] = make_grad_entry<0, 0, 2, 2, 2>();
  t[NGRADMODE * 6 + 0] = make_grad_entry<0, 1, 0, 0, 0>();
  t[NGRADMODE * 6 + 1] = make_grad_entry<0, 1, 0, 0, 2>();
  t[NGRADMODE * 7 + 0] = make_grad_entry<0, 1, 1, 0, 0>();
  t[NGRADMODE * 7 + 1] = make_grad_entry<0, 1, 1, 0, 2>();
  t[NGRADMODE * 8 + 0] = make_grad_entry<0, 1, 1, 1, 0>();
  t[NGRADMODE * 8 + 1] = make_grad_entry<0, 1, 1, 1, 2>();
  t[NGRADMODE * 9 + 0] = make_grad_entry<0, 1, 2, 0, 0>();
  t[NGRADMODE * 9 + 1] = make_grad_entry<0, 1, 2, 0, 2>();
  t[NGRADMODE * 10 + 0] = make_grad_entry<0, 1, 2, 1, 0>();
  t[NGRADMODE * 10 + 1] = make_grad_entry<0, 1, 2, 1, 2>();
  t[NGRADMODE * 11 + 0] = make_grad_entry<0, 1, 2, 2, 0>();
  t[NGRADMODE * 11 + 1] = make_grad_entry<0, 1, 2, 2, 2>();
  t[NGRADMODE * 12 + 0] = make_grad_entry<0, 2, 0, 0, 0>();
  t[NGRADMODE * 12 + 1] = make_grad_entry<0, 2, 0, 0, 2>();
  t[NGRADMODE * 13 + 0] = make_grad_entry<0, 2, 1, 0, 0>();
  t[NGRADMODE * 13 + 1] = make_grad_entry<0, 2, 1, 0, 2>();
  t[NGRADMODE * 14 + 0] = make_grad_entry<0, 2, 1, 1, 0>();
  t[NGRADMODE * 14 + 1] = make_grad_entry<0, 2, 1, 1, 2>();
  t[NGRADMODE * 15 + 0] = make_grad_entry<0, 2, 2, 0, 0>();
  t[NGRADMODE * 15 + 1] = make_grad_entry<0, 2, 2, 0, 2>();
  t[NGRADMODE * 16 + 0] = make_grad_entry<0, 2, 2, 1, 0>();
  t[NGRADMODE * 16 + 1] = make_grad_entry<0, 2, 2, 1, 2>();
  t[NGRADMODE * 17 + 0] = make_grad_entry<0, 2, 2, 2, 0>();
  t[NGRADMODE * 17 + 1] = make_grad_entry<0, 2, 2, 2, 2>();
}

}  // namespace lrb
