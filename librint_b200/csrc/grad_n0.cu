// Adjoint ERI kernels with the differentiated shell of momentum 0, centre modes (raised, lowered);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_n0(GradEntry *t) {
  t[NGRADMODE * 0 + 2] = make_grad_entry<0, 0, 0, 0, 1>();
  t[NGRADMODE * 1 + 2] = make_grad_entry<0, 0, 1, 0, 1>();
  t[NGRADMODE * 2 + 2] = make_grad_entry<0, 0, 1, 1, 1>();
  t[NGRADMODE * 3 + 2] = make_grad_entry<0, 0, 2, 0, 1>();
  t[NGRADMODE * 4 + 2] = make_grad_entry<0, 0, 2, 1, 1>();
  t[NGRADMODE * 5 + 2] = make_grad_entry<0, 0, 2, 2, 1>();
  t[NGRADMODE * 6 + 2] = make_grad_entry<0, 1, 0, 0, 1>();
  t[NGRADMODE * 7 + 2] = make_grad_entry<0, 1, 1, 0, 1>();
  t[NGRADMODE * 8 + 2] = make_grad_entry<0, 1, 1, 1, 1>();
  t[NGRADMODE * 9 + 2] = make_grad_entry<0, 1, 2, 0, 1>();
  t[NGRADMODE * 10 + 2] = make_grad_entry<0, 1, 2, 1, 1>();
  t[NGRADMODE * 11 + 2] = make_grad_entry<0, 1, 2, 2, 1>();
  t[NGRADMODE * 12 + 2] = make_grad_entry<0, 2, 0, 0, 1>();
  t[NGRADMODE * 13 + 2] = make_grad_entry<0, 2, 1, 0, 1>();
  t[NGRADMODE * 14 + 2] = make_grad_entry<0, 2, 1, 1, 1>();
  t[NGRADMODE * 15 + 2] = make_grad_entry<0, 2, 2, 0, 1>();
  t[NGRADMODE * 16 + 2] = make_grad_entry<0, 2, 2, 1, 1>();
  t[NGRADMODE * 17 + 2] = make_grad_entry<0, 2, 2, 2, 1>();
}

}  // namespace lrb
