// Adjoint ERI kernels with the differentiated shell of momentum 2, centre modes (raised, lowered);
// one TU per l so the kernels compile in parallel.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_n2(GradEntry *t) {
  t[NGRADMODE * 36 + 2] = make_grad_entry<2, 0, 0, 0, 1>();
  t[NGRADMODE * 36 + 3] = make_grad_entry<2, 0, 0, 0, 3>();
  t[NGRADMODE * 37 + 2] = make_grad_entry<2, 0, 1, 0, 1>();
  t[NGRADMODE * 37 + 3] = make_grad_entry<2, 0, 1, 0, 3>();
  t[NGRADMODE * 38 + 2] = make_grad_entry<2, 0, 1, 1, 1>();
  t[NGRADMODE * 38 + 3] = make_grad_entry<2, 0, 1, 1, 3>();
  t[NGRADMODE * 39 + 2] = make_grad_entry<2, 0, 2, 0, 1>();
  t[NGRADMODE * 39 + 3] = make_grad_entry<2, 0, 2, 0, 3>();
  t[NGRADMODE * 40 + 2] = make_grad_entry<2, 0, 2, 1, 1>();
  t[NGRADMODE * 40 + 3] = make_grad_entry<2, 0, 2, 1, 3>();
  t[NGRADMODE * 41 + 2] = make_grad_entry<2, 0, 2, 2, 1>();
  t[NGRADMODE * 41 + 3] = make_grad_entry<2, 0, 2, 2, 3>();
  t[NGRADMODE * 42 + 2] = make_grad_entry<2, 1, 0, 0, 1>();
  t[NGRADMODE * 42 + 3] = make_grad_entry<2, 1, 0, 0, 3>();
  t[NGRADMODE * 43 + 2] = make_grad_entry<2, 1, 1, 0, 1>();
  t[NGRADMODE * 43 + 3] = make_grad_entry<2, 1, 1, 0, 3>();
  t[NGRADMODE * 44 + 2] = make_grad_entry<2, 1, 1, 1, 1>();
  t[NGRADMODE * 44 + 3] = make_grad_entry<2, 1, 1, 1, 3>();
  t[NGRADMODE * 45 + 2] = make_grad_entry<2, 1, 2, 0, 1>();
  t[NGRADMODE * 45 + 3] = make_grad_entry<2, 1, 2, 0, 3>();
  t[NGRADMODE * 46 + 2] = make_grad_entry<2, 1, 2, 1, 1>();
  t[NGRADMODE * 46 + 3] = make_grad_entry<2, 1, 2, 1, 3>();
  t[NGRADMODE * 47 + 2] = make_grad_entry<2, 1, 2, 2, 1>();
  t[NGRADMODE * 47 + 3] = make_grad_entry<2, 1, 2, 2, 3>();
  t[NGRADMODE * 48 + 2] = make_grad_entry<2, 2, 0, 0, 1>();
  t[NGRADMODE * 48 + 3] = make_grad_entry<2, 2, 0, 0, 3>();
  t[NGRADMODE * 49 + 2] = make_grad_entry<2, 2, 1, 0, 1>();
  t[NGRADMODE * 49 + 3] = make_grad_entry<2, 2, 1, 0, 3>();
  t[NGRADMODE * 50 + 2] = make_grad_entry<2, 2, 1, 1, 1>();
  t[NGRADMODE * 50 + 3] = make_grad_entry<2, 2, 1, 1, 3>();
  t[NGRADMODE * 51 + 2] = make_grad_entry<2, 2, 2, 0, 1>();
  t[NGRADMODE * 51 + 3] = make_grad_entry<2, 2, 2, 0, 3>();
  t[NGRADMODE * 52 + 2] = make_grad_entry<2, 2, 2, 1, 1>();
  t[NGRADMODE * 52 + 3] = make_grad_entry<2, 2, 2, 1, 3>();
  t[NGRADMODE * 53 + 2] = make_grad_entry<2, 2, 2, 2, 1>();
  t[NGRADMODE * 53 + 3] = make_grad_entry<2, 2, 2, 2, 3>();
}

}  // namespace lrb
