// Adjoint ERI kernels with the differentiated shell of momentum 2 -- one TU per l.
#define RYS_OMIT_TAB
#define RYS_CONST_QUAL __constant__
#include "grad.h"

namespace lrb {

void grad_register_x2(GradEntry *t) {
  t[2 * 36 + 0] = make_grad_entry<2, 0, 0, 0, 0>();
  t[2 * 36 + 1] = make_grad_entry<2, 0, 0, 0, 2>();
  t[2 * 37 + 0] = make_grad_entry<2, 0, 1, 0, 0>();
  t[2 * 37 + 1] = make_grad_entry<2, 0, 1, 0, 2>();
  t[2 * 38 + 0] = make_grad_entry<2, 0, 1, 1, 0>();
  t[2 * 38 + 1] = make_grad_entry<2, 0, 1, 1, 2>();
  t[2 * 39 + 0] = make_grad_entry<2, 0, 2, 0, 0>();
  t[2 * 39 + 1] = make_grad_entry<2, 0, 2, 0, 2>();
  t[2 * 40 + 0] = make_grad_entry<2, 0, 2, 1, 0>();
  t[2 * 40 + 1] = make_grad_entry<2, 0, 2, 1, 2>();
  t[2 * 41 + 0] = make_grad_entry<2, 0, 2, 2, 0>();
  t[2 * 41 + 1] = make_grad_entry<2, 0, 2, 2, 2>();
  t[2 * 42 + 0] = make_grad_entry<2, 1, 0, 0, 0>();
  t[2 * 42 + 1] = make_grad_entry<2, 1, 0, 0, 2>();
  t[2 * 43 + 0] = make_grad_entry<2, 1, 1, 0, 0>();
  t[2 * 43 + 1] = make_grad_entry<2, 1, 1, 0, 2>();
  t[2 * 44 + 0] = make_grad_entry<2, 1, 1, 1, 0>();
  t[2 * 44 + 1] = make_grad_entry<2, 1, 1, 1, 2>();
  t[2 * 45 + 0] = make_grad_entry<2, 1, 2, 0, 0>();
  t[2 * 45 + 1] = make_grad_entry<2, 1, 2, 0, 2>();
  t[2 * 46 + 0] = make_grad_entry<2, 1, 2, 1, 0>();
  t[2 * 46 + 1] = make_grad_entry<2, 1, 2, 1, 2>();
  t[2 * 47 + 0] = make_grad_entry<2, 1, 2, 2, 0>();
  t[2 * 47 + 1] = make_grad_entry<2, 1, 2, 2, 2>();
  t[2 * 48 + 0] = make_grad_entry<2, 2, 0, 0, 0>();
  t[2 * 48 + 1] = make_grad_entry<2, 2, 0, 0, 2>();
  t[2 * 49 + 0] = make_grad_entry<2, 2, 1, 0, 0>();
  t[2 * 49 + 1] = make_grad_entry<2, 2, 1, 0, 2>();
  t[2 * 50 + 0] = make_grad_entry<2, 2, 1, 1, 0>();
  t[2 * 50 + 1] = make_grad_entry<2, 2, 1, 1, 2>();
  t[2 * 51 + 0] = make_grad_entry<2, 2, 2, 0, 0>();
  t[2 * 51 + 1] = make_grad_entry<2, 2, 2, 0, 2>();
  t[2 * 52 + 0] = make_grad_entry<2, 2, 2, 1, 0>();
  t[2 * 52 + 1] = make_grad_entry<2, 2, 2, 1, 2>();
  t[2 * 53 + 0] = make_grad_entry<2, 2, 2, 2, 0>();
  t[2 * 53 + 1] = make_grad_entry<2, 2, 2, 2, 2>();
}

}  // namespace lrb
