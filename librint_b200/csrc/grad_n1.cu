// Adjoint ERI kernels with the differentiated shell of momentum 1, centre modes (raised, lowered);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_n1(GradEntry *t) {
  t[NGRADMODE * 18 + 2] = make_grad_entry<1, 0, 0, 0, 1>();
  t[NGRADMODE * 18 + 3] = make_grad_entry<1, 0, 0, 0, 3>();
  t[NGRADMODE * 19 + 2] = make_grad_entry<1, 0, 1, 0, 1>();
  t[NGRADMODE * 19 + 3] = make_grad_entry<1, 0, 1, 0, 3>();
  t[NGRADMODE * 20 + 2] = make_grad_entry<1, 0, 1, 1, 1>();
  t[NGRADMODE * 20 + 3] = make_grad_entry<1, 0, 1, 1, 3>();
  t[NGRADMODE * 21 + 2] = make_grad_entry<1, 0, 2, 0, 1>();
  t[NGRADMODE * 21 + 3] = make_grad_entry<1, 0, 2, 0, 3>();
  t[NGRADMODE * 22 + 2] = make_grad_entry<1, 0, 2, 1, 1>();
  t[NGRADMODE * 22 + 3] = make_grad_entry<1, 0, 2, 1, 3>();
  t[NGRADMODE * 23 + 2] = make_grad_entry<1, 0, 2, 2, 1>();
  t[NGRADMODE * 23 + 3] = make_grad_entry<1, 0, 2, 2, 3>();
  t[NGRADMODE * 24 + 2] = make_grad_entry<1, 1, 0, 0, 1>();
  t[NGRADMODE * 24 + 3] = make_grad_entry<1, 1, 0, 0, 3>();
  t[NGRADMODE * 25 + 2] = make_grad_entry<1, 1, 1, 0, 1>();
  t[NGRADMODE * 25 + 3] = make_grad_entry<1, 1, 1, 0, 3>();
  t[NGRADMODE * 26 + 2] = make_grad_entry<1, 1, 1, 1, 1>();
  t[NGRADMODE * 26 + 3] = make_grad_entry<1, 1, 1, 1, 3>();
  t[NGRADMODE * 27 + 2] = make_grad_entry<1, 1, 2, 0, 1>();
  t[NGRADMODE * 27 + 3] = make_grad_entry<1, 1, 2, 0, 3>();
  t[NGRADMODE * 28 + 2] = make_grad_entry<1, 1, 2, 1, 1>();
  t[NGRADMODE * 28 + 3] = make_grad_entry<1, 1, 2, 1, 3>();
  t[NGRADMODE * 29 + 2] = make_grad_entry<1, 1, 2, 2, 1>();
  t[NGRADMODE * 29 + 3] = make_grad_entry<1, 1, 2, 2, 3>();
  t[NGRADMODE * 30 + 2] = make_grad_entry<1, 2, 0, 0, 1>();
  t[NGRADMODE * 30 + 3] = make_grad_entry<1, 2, 0, 0, 3>();
  t[NGRADMODE * 31 + 2] = make_grad_entry<1, 2, 1, 0, 1>();
  t[NGRADMODE * 31 + 3] = make_grad_entry<1, 2, 1, 0, 3>();
  t[NGRADMODE * 32 + 2] = make_grad_entry<1, 2, 1, 1, 1>();
  t[NGRADMODE * 32 + 3] = make_grad_entry<1, 2, 1, 1, 3>();
  t[NGRADMODE * 33 + 2] = make_grad_entry<1, 2, 2, 0, 1>();
  t[NGRADMODE * 33 + 3] = make_grad_entry<1, 2, 2, 0, 3>();
  t[NGRADMODE * 34 + 2] = make_grad_entry<1, 2, 2, 1, 1>();
  t[NGRADMODE * 34 + 3] = make_grad_entry<1, 2, 2, 1, 3>();
  t[NGRADMODE * 35 + 2] = make_grad_entry<1, 2, 2, 2, 1>();
  t[NGRADMODE * 35 + 3] = make_grad_entry<1, 2, 2, 2, 3>();
}

}  // namespace lrb
