/* Oracle: CPU restatement of librint's Rys-ERI / RHF path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code: only tests/, __graft_entry__.smoke() (as the checker) and
 * bench.py's cpu_baseline / --impl reference leg use it.
 *
 * Parity pins: the oracle is checked against golden vectors produced by the
 * reference's own shipped library (tests/golden/make_golden.py), against the
 * energy truths in checks/truth/{h2,h2o}/sto3g_E.txt, and its Rys tables
 * against 60-digit mpmath rules and against its own binary128 rules
 * (orc_set_rys_mode), which share no table, generator or algorithm with the
 * CUDA kernels.
 *
 * Array conventions are librint's (src/p2c.rs, src/scf.rs): atm has 6 ints per
 * atom, bas 8 ints per shell, env holds coordinates, exponents and PySCF-
 * normalised contraction coefficients.  Matrices are row-major n x n in AO
 * order; coord = 0 cartesian, 1 spherical.
 */
#ifndef LIBRINT_ORACLE_H
#define LIBRINT_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Rys nodes u = t^2/(1-t^2) and weights for nroots n (1..9) at x. */
void orc_rys_roots(int n, double x, double *u, double *w);
/* Source of every Rys rule the oracle uses from now on: 0 (default) the
 * tables the CUDA kernels also read, 1 a binary128 Gauss rule computed from
 * the measure (no shared table or generator; about 1 ms per rule). */
void orc_set_rys_mode(int mode);

/* One shell quartet, libcint layout out[i + ni*(j + nj*(k + nk*l))].
 * Returns 1 if any primitive quartet survived screening, else 0 (out zeroed).
 * Follows src/eri.rs:409-516 with the screening of src/cint2e.rs:36-465. */
int orc_int2e_cart(double *out, const int *shls, const int *atm, int natm,
                   const int *bas, int nbas, const double *env);
int orc_int2e_sph(double *out, const int *shls, const int *atm, int natm,
                  const int *bas, int nbas, const double *env);

/* Many independent quartets (shls[4*q..4*q+3]); the blocks are packed back to
 * back in quartet order.  OpenMP over quartets with nthreads threads. */
void orc_int2e_batch(double *out, int coord, const int *shls, long nq,
                     const int *atm, int natm, const int *bas, int nbas,
                     const double *env, int nthreads);

/* Dense n^4 tensor R[((mu*n+nu)*n+sig)*n+lam] (src/scf.rs:215-311). */
void orc_int2e_tensor(double *out, int coord, const int *atm, int natm,
                      const int *bas, int nbas, const double *env, int nthreads);

/* One-electron matrix: typec 0 overlap, 1 kinetic, 2 nuclear attraction
 * (src/scf.rs:149-213). */
void orc_int1e(double *out, int coord, int typec, const int *atm, int natm,
               const int *bas, int nbas, const double *env);

/* Direct two-electron Fock part G(P), full nbas^4 loop (src/scf.rs:316-410).*/
void orc_fock_G(double *G, const double *P, int coord, const int *atm, int natm,
                const int *bas, int nbas, const double *env, int nthreads);

/* The same digestion over a given list of shell quartets (shls[4*q..]),
 * each visited once in the reference's slot order -- a bounded sample of
 * the nbas^4 loop for timing. */
void orc_fock_G_quartets(double *G, const double *P, const int *shls, long nq,
                         const int *atm, int natm, const int *bas, int nbas,
                         const double *env, int nthreads);

/* G restricted to shell-pair blocks (X, Y) = pairs[2p], pairs[2p+1]: every
 * term of the reference's nbas^4 digestion that lands in G[mu in X, nu in Y],
 * summed exactly; blocks packed back to back, row-major (mu, nu).  Cost
 * 2 nbas^2 quartets per block, so it checks large molecules block-wise. */
void orc_fock_G_blocks(double *out, const double *P, const int *pairs, int npairs,
                       const int *atm, int natm, const int *bas, int nbas,
                       const double *env, int nthreads);

/* 1/2 sum P G(P) over the unique quartets (8-fold symmetry, degeneracy
 * weights), and the one-electron plus nuclear part sum P (T + V) + E_nn:
 * their sum is the reference's energy functional (src/scf.rs:827-956). */
double orc_energy2_sym(const double *P, const int *atm, int natm, const int *bas,
                       int nbas, const double *env, int nthreads);
double orc_energy1(const double *P, const int *atm, int natm, const int *bas, int nbas,
                   const double *env);

/* RHF in the cartesian basis (src/scf.rs:743-969).  density returns 0 on
 * success, 1 near-singular S, 2 not converged, 3 invalid density. */
int orc_density(double *P, size_t nelec, int imax, double conv,
                const int *atm, int natm, const int *bas, int nbas,
                const double *env, int nthreads, int *iters);
double orc_energy(const double *P, const int *atm, int natm, const int *bas,
                  int nbas, const double *env, int nthreads);
double orc_scf(size_t nelec, int imax, double conv, const int *atm, int natm,
               const int *bas, int nbas, const double *env, int nthreads);

/* Number of AOs (coord 0 cart, 1 sph), nctr included (src/scf.rs:136-151). */
int orc_nao(int coord, const int *bas, int nbas);

#ifdef __cplusplus
}
#endif
#endif
