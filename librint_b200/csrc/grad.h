// Gradient driver and adjoint-kernel class table (see grad.cu).
#pragma once
#include <cublas_v2.h>

#include "fock.h"
#include "grad_kernel.cuh"

namespace lrb {

// gradient classes: X (differentiated, first) and its pair partner Y in
// any order (3 x 3), the other pair in table orientation (6 pair classes)
constexpr int NGRADCLS = 54;

using GradKernelFn = void (*)(GradParams, const double *, int *);
struct GradEntry {
  GradKernelFn fn;
  size_t smem;
  int slots, nr;
};

template <int LX, int LY, int LZ, int LW, int MODE>
GradEntry make_grad_entry() {
  using C = EriClass<LX + grad_dl(MODE), LY, LZ, LW>;
  GradEntry e;
  e.fn = k_eri_grad<LX, LY, LZ, LW, MODE>;
  e.smem = GradLayout<C, grad_nc(MODE)>::SMEM;
  e.slots = C::SLOTS;
  e.nr = C::NR;
  return e;
}

// t is GradEntry[NGRADCLS][NGRADMODE], mode slots 0..3 = modes 0, 2, 1, 3
// (coefficient, exponent, centre raised, centre lowered; the last is absent
// for l_X = 0); id = (lx*3 + ly)*6 + ket pair class.  The x units register
// the environment modes, the n units the centre modes.
constexpr int NGRADMODE = 4;
void grad_register_x0(GradEntry *t);
void grad_register_x1(GradEntry *t);
void grad_register_x2(GradEntry *t);
void grad_register_n0(GradEntry *t);
void grad_register_n1(GradEntry *t);
void grad_register_n2(GradEntry *t);

cublasHandle_t grad_blas();
// d_grad[t] += cH dH + cR dR + cS dS for env[s1 + t]; d_P on the device.
int grad_run(MolCtx &m, const double *d_P, double cH, double cR, double cS, double tau,
             double *d_grad, int s1, cudaStream_t st);
// d_gatom[3 * atom + axis] += d/dR of the RHF energy at the converged
// density d_P: dH + dR - (1/2) sum (P F P) dS + d E_nuc (all on the device).
int grad_nuc_run(MolCtx &m, const double *d_P, double tau, double *d_gatom, cudaStream_t st);
// Full env Jacobian of S (op 0), T (1) or V (2): d_out[(nu n + mu) nenv + l].
int d1e_env_run(MolCtx &m, int op, double *d_out, cudaStream_t st);
// Overlap Jacobian d S[mu nu] / d env[s1 + l] into d_out[(nu n + mu) L + l].
int dS_u_run(MolCtx &m, int s1, int L, double *d_out, cudaStream_t st);

}  // namespace lrb
