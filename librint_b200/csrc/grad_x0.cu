// Adjoint ERI kernels with the differentiated shell of momentum 0 -- one TU per l.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x0(GradEntry *t) {
  t[2 * 0 + 0] = make_grad_entry<0, 0, 0, 0, 0>();
  t[2 * 0 + 1] = make_grad_entry<0, 0, 0, 0, 2>();
  t[2 * 1 + 0] = make_grad_entry<0, 0, 1, 0, 0>();
  t[2 * 1 + 1] = make_grad_entry<0, 0, 1, 0, 2>();
  t[2 * 2 + 0] = make_grad_entry<0, 0, 1, 1, 0>();
  t[2 * 2 + 1] = make_grad_entry<0, 0, 1, 1, 2>();
  t[2 * 3 + 0] = make_grad_entry<0, 0, 2, 0, 0>();
  t[2 * 3 + 1] = make_grad_entry<0, 0, 2, 0, 2>();
  t[2 * 4 + 0] = make_grad_entry<0, 0, 2, 1, 0>();
  t[2 * 4 + 1] = make_grad_entry<0, 0, 2, 1, 2>();
  t[2 * 5 + 0] = make_grad_entry<0, 0, 2, 2, 0>();
  t[2 * 5 + 1] = make_grad_entry<0, 0, 2, 2, 2>();
  t[2 * 6 + 0] = make_grad_entry<0, 1, 0, 0, 0>();
  t[2 * 6 + 1] = make_grad_entry<0, 1, 0, 0, 2>();
  t[2 * 7 + 0] = make_grad_entry<0, 1, 1, 0, 0>();
  t[2 * 7 + 1] = make_grad_entry<0, 1, 1, 0, 2>();
  t[2 * 8 + 0] = make_grad_entry<0, 1, 1, 1, 0>();
  t[2 * 8 + 1] = make_grad_entry<0, 1, 1, 1, 2>();
  t[2 * 9 + 0] = make_grad_entry<0, 1, 2, 0, 0>();
  t[2 * 9 + 1] = make_grad_entry<0, 1, 2, 0, 2>();
  t[2 * 10 + 0] = make_grad_entry<0, 1, 2, 1, 0>();
  t[2 * 10 + 1] = make_grad_entry<0, 1, 2, 1, 2>();
  t[2 * 11 + 0] = make_grad_entry<0, 1, 2, 2, 0>();
  t[2 * 11 + 1] = make_grad_entry<0, 1, 2, 2, 2>();
  t[2 * 12 + 0] = make_grad_entry<0, 2, 0, 0, 0>();
  t[2 * 12 + 1] = make_grad_entry<0, 2, 0, 0, 2>();
  t[2 * 13 + 0] = make_grad_entry<0, 2, 1, 0, 0>();
  t[2 * 13 + 1] = make_grad_entry<0, 2, 1, 0, 2>();
  t[2 * 14 + 0] = make_grad_entry<0, 2, 1, 1, 0>();
  t[2 * 14 + 1] = make_grad_entry<0, 2, 1, 1, 2>();
  t[2 * 15 + 0] = make_grad_entry<0, 2, 2, 0, 0>();
  t[2 * 15 + 1] = make_grad_entry<0, 2, 2, 0, 2>();
  t[2 * 16 + 0] = make_grad_entry<0, 2, 2, 1, 0>();
  t[2 * 16 + 1] = make_grad_entry<0, 2, 2, 1, 2>();
  t[2 * 17 + 0] = make_grad_entry<0, 2, 2, 2, 0>();
  t[2 * 17 + 1] = make_grad_entry<0, 2, 2, 2, 2>();
}

}  // namespace lrb
