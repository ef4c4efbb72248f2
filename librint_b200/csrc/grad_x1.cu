// Adjoint ERI kernels with the differentiated shell of momentum 1 -- one TU per l.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x1(GradEntry *t) {
  t[2 * 18 + 0] = make_grad_entry<1, 0, 0, 0, 0>();
  t[2 * 18 + 1] = make_grad_entry<1, 0, 0, 0, 2>();
  t[2 * 19 + 0] = make_grad_entry<1, 0, 1, 0, 0>();
  t[2 * 19 + 1] = make_grad_entry<1, 0, 1, 0, 2>();
  t[2 * 20 + 0] = make_grad_entry<1, 0, 1, 1, 0>();
  t[2 * 20 + 1] = make_grad_entry<1, 0, 1, 1, 2>();
  t[2 * 21 + 0] = make_grad_entry<1, 0, 2, 0, 0>();
  t[2 * 21 + 1] = make_grad_entry<1, 0, 2, 0, 2>();
  t[2 * 22 + 0] = make_grad_entry<1, 0, 2, 1, 0>();
  t[2 * 22 + 1] = make_grad_entry<1, 0, 2, 1, 2>();
  t[2 * 23 + 0] = make_grad_entry<1, 0, 2, 2, 0>();
  t[2 * 23 + 1] = make_grad_entry<1, 0, 2, 2, 2>();
  t[2 * 24 + 0] = make_grad_entry<1, 1, 0, 0, 0>();
  t[2 * 24 + 1] = make_grad_entry<1, 1, 0, 0, 2>();
  t[2 * 25 + 0] = make_grad_entry<1, 1, 1, 0, 0>();
  t[2 * 25 + 1] = make_grad_entry<1, 1, 1, 0, 2>();
  t[2 * 26 + 0] = make_grad_entry<1, 1, 1, 1, 0>();
  t[2 * 26 + 1] = make_grad_entry<1, 1, 1, 1, 2>();
  t[2 * 27 + 0] = make_grad_entry<1, 1, 2, 0, 0>();
  t[2 * 27 + 1] = make_grad_entry<1, 1, 2, 0, 2>();
  t[2 * 28 + 0] = make_grad_entry<1, 1, 2, 1, 0>();
  t[2 * 28 + 1] = make_grad_entry<1, 1, 2, 1, 2>();
  t[2 * 29 + 0] = make_grad_entry<1, 1, 2, 2, 0>();
  t[2 * 29 + 1] = make_grad_entry<1, 1, 2, 2, 2>();
  t[2 * 30 + 0] = make_grad_entry<1, 2, 0, 0, 0>();
  t[2 * 30 + 1] = make_grad_entry<1, 2, 0, 0, 2>();
  t[2 * 31 + 0] = make_grad_entry<1, 2, 1, 0, 0>();
  t[2 * 31 + 1] = make_grad_entry<1, 2, 1, 0, 2>();
  t[2 * 32 + 0] = make_grad_entry<1, 2, 1, 1, 0>();
  t[2 * 32 + 1] = make_grad_entry<1, 2, 1, 1, 2>();
  t[2 * 33 + 0] = make_grad_entry<1, 2, 2, 0, 0>();
  t[2 * 33 + 1] = make_grad_entry<1, 2, 2, 0, 2>();
  t[2 * 34 + 0] = make_grad_entry<1, 2, 2, 1, 0>();
  t[2 * 34 + 1] = make_grad_entry<1, 2, 2, 1, 2>();
  t[2 * 35 + 0] = make_grad_entry<1, 2, 2, 2, 0>();
  t[2 * 35 + 1] = make_grad_entry<1, 2, 2, 2, 2>();
}

}  // namespace lrb
