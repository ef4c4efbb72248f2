/* librint_b200: B200 (sm_100a) Rys-quadrature ERIs and RHF Fock builds behind
 * librint's C ABI.
 *
 * Array conventions are librint's / libcint's: atm has 6 int32 slots per atom,
 * bas 8 int32 slots per shell, env is the float64 pool they index into
 * (reference src/p2c.rs:1-15).  coord = 0 cartesian, 1 spherical.
 * Matrices are row-major n x n in AO order; ERI blocks are column-major
 * (i fastest) like libcint.
 *
 * Errors: entry points of this library's own API return a status code
 * (LRB_OK or a negative LRB_ERR_*); lrb_last_error() describes the last
 * failure on the calling thread.  The reference-shaped entry points keep the
 * reference's in-band conventions (NULL / NaN) and never exit the process.
 *
 * Threads: the library keeps one set of streams and device workspaces per
 * device, shared by every call on that device; calls on one device from
 * several host threads must not overlap (each call works on the device that
 * is current on its thread).
 */
#ifndef LIBRINT_B200_H
#define LIBRINT_B200_H
#include <stddef.h>

#if defined(__GNUC__)
#define LRB_API __attribute__((visibility("default")))
#else
#define LRB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define LRB_OK 0
#define LRB_ERR_INPUT (-1)
#define LRB_ERR_UNSUPPORTED (-2)
#define LRB_ERR_ALLOC (-3)
#define LRB_ERR_CUDA (-4)
#define LRB_ERR_SCF (-5)
#define LRB_ERR_TIMEOUT (-6)

/* Text of the last error on this thread ("" if none). */
LRB_API const char *lrb_last_error(void);

/* ---------------------------------------------------------------------
 * Batched shell-quartet ERIs -- the GPU entry for the per-quartet loops of
 * src/scf.rs:102-118 (Basis::int2e) and src/scf.rs:253-307 (integral2e),
 * each iteration of which calls cint2e_sph / cint2e_cart
 * (src/cint2e.rs:2896, 2938).
 *
 * shls holds nq quartets (4 shell indices each).  Every quartet's block is
 * written in libcint layout (out[i + ni*(j + nj*(k + nk*l))]) and the blocks
 * are packed back to back in quartet order; lrb_int2e_batch_len gives the
 * total length in doubles.  Shells: l <= 3 with 1..31 primitives.
 * Generally contracted shells (nctr > 1; blocks of nf * nctr rows per shell,
 * contraction-major as libcint) are accepted by lrb_int2e_batch, which splits
 * them into segmented sub-shells on the host; the device-pointer entry points
 * take segmented shells only.  Screening is the reference's (expcutoff from
 * env[0], 60 by default, src/cint2e.rs:367-393); env[8] = omega selects the
 * range-separated operator (src/g2e.rs:5564-5612).
 * -------------------------------------------------------------------*/
LRB_API long long lrb_int2e_batch_len(int coord, const int *shls, long long nq, const int *bas, int nbas);

/* Host pointers; copies in, computes on the current device, copies out.
 * The indices and bas entries are checked on up to 32 host threads before
 * any device work; the quartets then run in chunks whose copies in and out
 * overlap other chunks' kernels when out (and the inputs) are page-locked.
 * Returns after the whole output is on the host. */
LRB_API int lrb_int2e_batch(double *out, int coord, const int *shls, long long nq, const int *atm,
                    int natm, const int *bas, int nbas, const double *env, long long nenv);

/* Device pointers; asynchronous on `stream` (a cudaStream_t, NULL = legacy
 * default stream).  Returns after the work is queued. */
LRB_API int lrb_int2e_batch_device(double *out, int coord, const int *shls, long long nq,
                           const int *atm, int natm, const int *bas, int nbas,
                           const double *env, long long nenv, void *stream);

/* lrb_int2e_batch_device for callers that may not allocate device memory
 * (a framework whose caching allocator already holds the free memory, or a
 * latency-bound loop that cannot take cudaMalloc's device synchronisation).
 * No counterpart in the reference.  All scratch comes from one static device
 * array of LRB_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds
 * until exit.  Batches over LRB_NOALLOC_MAX_QUARTETS quartets, or whose
 * quartet tables plus primitive pairs (128 bytes per pair, bra and ket) do not
 * fit, are rejected with LRB_ERR_INPUT and the sizes in lrb_last_error().
 * Calls share the array: each clears what must start at zero itself, and
 * calls whose GPU work overlaps race.  The first call on a device sets up
 * (symbol lookup, kernel table); make it before any stream capture.  Under
 * CUDA's default lazy module loading the array is placed in device memory at
 * that first call, so make it (a warm-up call will do) before other code
 * reserves the GPU's free memory, or set CUDA_MODULE_LOADING=EAGER.  A call
 * synchronises `stream` three times while preparing the batch. */
#define LRB_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define LRB_NOALLOC_MAX_QUARTETS 65536
LRB_API int lrb_int2e_batch_device_noalloc(double *out, int coord, const int *shls, long long nq,
                                           const int *atm, int natm, const int *bas, int nbas,
                                           const double *env, long long nenv, void *stream);

/* Measurement hooks (no reference counterpart).  While enabled, every ERI
 * class kernel is bracketed by CUDA events on its stream; lrb_profile_read
 * adds the milliseconds per class id (canonical order (ss|ss), (ps|ss),
 * (ps|ps), (pp|ss), ... (dd|dd)) into ms[0..n) and returns the number of
 * kernels harvested.  lrb_launch_count counts this library's kernel
 * launches; lrb_fp64_peak_probe measures FP64 FMA throughput (TFLOP/s). */
LRB_API void lrb_profile_enable(int on);
LRB_API int lrb_profile_read(double *ms, int n);
/* Fock builds run while profiling: per Fock class id (canonical class id,
 * plus 55 for the FP32 kernels) the shell quartets and the primitive
 * quartets that passed screening, since the last read (which clears them). */
LRB_API int lrb_fock_class_counts(long long *quartets, long long *prim_quartets, int n);
/* Fock builds: shell quartets of the small classes (at most 27 cartesian
 * elements, (ss|ss) ... (dp|ss); also (ds|pp), (ds|ds) and, FP64, (pp|pp))
 * with at least kmin primitive quartets run one lane per primitive quartet
 * instead of one slot per shell quartet.  kmin > 0
 * sets the bound for the process (default 32, or LRB_FOCK_LP_MIN; 1048576
 * disables those kernels); every call returns the bound in force. */
LRB_API int lrb_fock_lane_min(int kmin);
LRB_API long long lrb_launch_count(void);
LRB_API double lrb_fp64_peak_probe(int ms);

/* ---------------------------------------------------------------------
 * libcint per-quartet ABI (src/cint2e.rs:2896 int2e_sph, :2938 int2e_cart,
 * :2927 int2e_optimizer; src/optimizer.rs:81 CINTdel_optimizer).
 * out == NULL returns the scratch size in doubles (this implementation
 * needs none and returns the block size); dims == NULL means a packed
 * block; cache is ignored.  Returns 1 if the block is non-zero, else 0.
 * An optimizer keeps device copies of atm/bas/env for later calls.
 * -------------------------------------------------------------------*/
typedef struct LrbCintOpt CINTOpt;
LRB_API int int2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
              double *env, CINTOpt *opt, double *cache);
LRB_API int int2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
               double *env, CINTOpt *opt, double *cache);
LRB_API void int2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);
LRB_API void CINTdel_optimizer(CINTOpt **opt);

/* ---------------------------------------------------------------------
 * librint C ABI (src/p2c.rs).  Inputs are read as (pointer, element count)
 * pairs and not retained.  Returned buffers are malloc'd and must be
 * released with free_c(ptr, len) (src/p2c.rs:68).
 * -------------------------------------------------------------------*/
LRB_API void free_c(double *ptr, size_t len);

/* Dense n^4 ERI tensor R[((mu*n+nu)*n+sig)*n+lam] (src/p2c.rs:109,
 * src/scf.rs:215-311); NULL on failure. */
LRB_API double *int2e_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                size_t env_l, int coord);

/* ---------------------------------------------------------------------
 * Molecule context, direct Fock build and SCF on the GPU.
 * A context holds device copies of atm/bas/env, the shell-pair table with
 * primitive-pair data and Schwarz factors; it is reused across Fock builds.
 * Matrices are n x n (cartesian AOs, the reference's SCF basis).
 * -------------------------------------------------------------------*/
typedef struct LrbMol LrbMol;
LRB_API int lrb_mol_create(LrbMol **out, const int *atm, int natm, const int *bas, int nbas,
                           const double *env, long long nenv);
LRB_API void lrb_mol_destroy(LrbMol *m);
LRB_API int lrb_mol_nao(const LrbMol *m);

/* G(P) = J - K/2 without the n^4 tensor -- the GPU form of integral2e_fock
 * (src/scf.rs:316-410).  Quartets with Q_IJ Q_KL max|D| < tau are skipped
 * (tau = 0 keeps every quartet the reference keeps).  Host or device. */
LRB_API int lrb_fock_G(LrbMol *m, const double *P, double *G, double tau, long long *quartets);
LRB_API int lrb_fock_G_device(LrbMol *m, const double *P, double *G, double tau, void *stream);
/* One rank's share of G(P) for a Fock build split over nranks GPUs (no
 * reference counterpart; the reference's integral2e_fock, src/scf.rs:316-410,
 * is serial): the screened quartet candidates are enumerated in one order
 * fixed by the Schwarz-sorted shell pairs, and rank r digests the candidates
 * whose index is r mod nranks.  The shares are disjoint and complete, so the
 * sum over ranks (one all-reduce of n*n doubles) is lrb_fock_G's G.  Host
 * buffers, or device buffers on `stream` (_device). */
LRB_API int lrb_fock_G_part(LrbMol *m, const double *P, double *G, double tau, int rank,
                            int nranks, long long *quartets);
LRB_API int lrb_fock_G_part_device(LrbMol *m, const double *P, double *G, double tau, int rank,
                                   int nranks, long long *quartets, void *stream);
/* The same G(P) with the mixed-precision kernels (no reference counterpart):
 * prec 0 all FP64, 1 all FP32, 2 FP32 only for quartets whose Schwarz x
 * density bound is below tau32.  FP32 quartets run the recurrences and the
 * digestion in FP32 (roots, weights and prefactors FP64, rounded once) and
 * add into FP64 J/K.  Host
 * buffers; quartets / fp32_quartets (may be NULL) receive the counts. */
LRB_API int lrb_fock_G_prec(LrbMol *m, const double *P, double *G, double tau, int prec,
                            double tau32, long long *quartets, long long *fp32_quartets);

typedef struct {
  int max_iter;       /* reference imax */
  double conv;        /* reference conv: ||P - P_old||_F / 2 */
  int guess;          /* 0: P0 = I (reference), 1: core Hamiltonian */
  int diis;           /* DIIS subspace, at most 20 (0 = plain Roothaan, as the reference) */
  double tau;         /* quartet screening threshold */
  int mixed;          /* 1: incremental Fock builds, FP32 for small quartets */
  double fp32_until;  /* all-FP32 builds while ||dP|| is above this */
  double tau32;       /* then FP32 only for Schwarz x |dD| bounds below this */
  int rebuild_every;  /* full (non-incremental) Fock build period */
  double tau_fp32;    /* screening threshold of the FP32 and split builds
                         (0: tau); the FP64 phase always screens at tau */
  double tau_prim;    /* primitive-quartet screening of the Fock builds (0: off;
                         see lrb_mol_set_tau_prim) */
} LrbScfOptions;

typedef struct {
  double energy, e_nuc, delta, fock_ms, wall_ms;
  int iterations, converged;
  long long quartets, fp32_quartets;
} LrbScfResult;

/* Primitive-quartet screening of a context's Fock builds (no reference
 * counterpart; the reference screens primitives only by its exponent test,
 * src/cint2e.rs:367-393): a primitive quartet of a kept shell quartet is
 * skipped when Q_ij Q_kl d < tau_prim, Q the primitive pairs' Schwarz factors
 * sqrt(max |(ij|ij)|) and d the shell quartet's density factor.  FP32 quartets
 * use the larger of tau_prim and the build's quartet threshold.  0 (the
 * default) keeps every primitive quartet the reference keeps. */
LRB_API int lrb_mol_set_tau_prim(LrbMol *m, double tau_prim);

/* RHF (src/scf.rs:743-969).  P_out (n*n host) and P0 (initial density,
 * overrides guess) may be NULL. */
LRB_API int lrb_scf(LrbMol *m, long long nelec, const LrbScfOptions *opt, LrbScfResult *res,
                    double *P_out, const double *P0);
/* Energy functional at a density (src/scf.rs:827-956, energyfast). */
LRB_API int lrb_energy(LrbMol *m, const double *P, double tau, double *E);
/* One-electron matrix: typec 0 overlap, 1 kinetic, 2 nuclear (src/scf.rs:149). */
LRB_API int lrb_int1e(LrbMol *m, int typec, int coord, double *out);

/* librint p2c.rs entry points (src/p2c.rs:86, 153, 186, 210). */
LRB_API double *int1e_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                        size_t env_l, int coord, int typec);
LRB_API double *density_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                          size_t env_l, size_t nelec, int imax, double conv);
LRB_API double energy_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                        size_t env_l, double *P_p, size_t P_l);
LRB_API double scf_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                     size_t env_l, size_t nelec, int imax, double conv);

/* ---------------------------------------------------------------------
 * Frozen-density gradient with respect to env[s1:s2] -- the exponents and
 * contraction coefficients (src/utils.rs:152-175 split, src/dscf.rs:320-565):
 *   out = cH dH + cR dR + cS dS,  dH = sum P (dT + dV),
 *   dR = d/dtheta 1/2 sum (P P - P P / 2)(ij|kl),  dS = sum (P F P) dS.
 * dR comes from an adjoint ERI kernel contracted with the density in-kernel
 * (replacing the Enzyme reverse passes of src/dscf.rs:370-515).
 * -------------------------------------------------------------------*/
LRB_API int lrb_grad_len(const LrbMol *m);
LRB_API int lrb_grad(LrbMol *m, const double *P, double cH, double cR, double cS, double tau,
                     double *out);

/* RHF gradient with respect to the nuclear coordinates, out[3*atom + axis]
 * (natm*3 doubles, Hartree/Bohr), at a converged density P (n*n host):
 *   dE/dR = sum P dH/dR + dR/dR - 1/2 sum (P F P) dS/dR + dE_nuc/dR,
 * with the nuclear-attraction Hellmann-Feynman term and the ERI centre
 * derivatives contracted in-kernel (2 a x^(a+1) - a_d x^(a-1) per primitive).
 * The reference differentiates only exponents and coefficients
 * (src/utils.rs:152-175); the coordinates are this library's extension. */
LRB_API int lrb_grad_nuc(LrbMol *m, const double *P, double tau, double *out);

/* Full Jacobian of a one-electron matrix (typec 0 S, 1 T, 2 V) with respect
 * to every env entry -- coordinates (including, for V, the nuclei of the
 * operator), exponents and coefficients: out[(nu*n + mu)*nenv + l] =
 * d O[mu nu] / d env[l], n*n*nenv doubles (host).  The reference computes the
 * same Jacobians with Enzyme in its checks (checks/overlap.rs:96-175,
 * kinetic.rs, nuclear.rs); there is no reference ABI counterpart. */
LRB_API int lrb_int1e_jacobian(LrbMol *m, int typec, double *out);

/* src/p2c.rs:131 dS_u: overlap Jacobian with respect to env[s1:s2]
 * (src/dscf.rs:96-151); element (nu * n + mu) * L + l = d S[mu nu] /
 * d env[s1 + l], n*n*L doubles (n cartesian AOs, L = s2 - s1); free_c. */
LRB_API double *dS_u(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                     size_t env_l);

/* src/p2c.rs:240, 267, 294, 321, 348, 376: buffers of lrb_grad_len doubles,
 * release with free_c; NULL on failure. */
LRB_API double *grad_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                       size_t env_l, double *P_p, size_t P_l);
LRB_API double *dS_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                     size_t env_l, double *P_p, size_t P_l);
LRB_API double *dHcore_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                         size_t env_l, double *P_p, size_t P_l);
LRB_API double *dR_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                     size_t env_l, double *P_p, size_t P_l);
LRB_API double *danalytical_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l,
                              double *env_p, size_t env_l, double *P_p, size_t P_l);
LRB_API double *denergy_c(int *atm_p, size_t atm_l, int *bas_p, size_t bas_l, double *env_p,
                          size_t env_l, double *P_p, size_t P_l);

/* ---------------------------------------------------------------------
 * Learned initial guess: MLP kernels (FP32, device pointers, async on
 * `stream`).  No reference counterpart (the reference starts from P = I,
 * src/scf.rs:757-764).  A layer is Y = act(X W^T + b), X (M x K), W (N x K);
 * act 0 identity, 1 SiLU.
 * -------------------------------------------------------------------*/
LRB_API int lrb_mlp_forward(const float *X, int M, int K, const float *W, const float *b, int N,
                            int act, float *Z, float *Y, void *stream);
LRB_API int lrb_mlp_backward(const float *X, int M, int K, const float *W, int N, int act,
                             const float *Z, const float *dY, float *dZ, float *dW, float *db,
                             float *dX, void *stream);
LRB_API int lrb_mse(const float *Y, const float *T, const float *Wt, long long n, float inv_count,
                    float *dY, float *loss, void *stream);
LRB_API int lrb_adam(float *p, const float *g, float *m, float *v, long long n, float lr,
                     float b1, float b2, float eps, int step, void *stream);

#ifdef __cplusplus
}
#endif
#endif
