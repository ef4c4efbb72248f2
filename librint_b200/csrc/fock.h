// Molecule context and direct Fock build (see fock.cu).
#pragma once
#include <vector>

#include "engine.h"
#include "eri_device.cuh"

namespace lrb {

struct MolCtx {
  int natm = 0, nbas = 0, nao = 0, npairs = 0, npp = 0;
  int gc = 0;   // built from generally contracted shells (h_bas holds the sub-shells)
  long long nenv = 0;
  std::vector<int> h_atm, h_bas, h_aooff;
  std::vector<double> h_env;
  std::vector<PairInfo> h_pairs;
  int *atm = nullptr, *bas = nullptr, *aooff = nullptr, *pcls = nullptr;
  double *env = nullptr, *Q = nullptr, *Dsh = nullptr;
  double *centers = nullptr;   // 3 doubles per shell
  PairInfo *pairs = nullptr;
  PrimPair *pp = nullptr;    // primitive pairs of each table pair, ip fastest
  // pairs by descending Schwarz factor: qorder[position] = pair, Qs = Q sorted;
  // per-position candidate counts / offsets and the density maximum of a build
  int *qorder = nullptr, *qcnt = nullptr;
  double *Qs = nullptr, *dmax = nullptr;
  long long *qoff = nullptr;
  // log Schwarz factor of every primitive pair (same order as pp), and the
  // primitive-quartet screening threshold of this context's Fock builds
  // (0: only the reference's exponent screening)
  float *lq = nullptr;
  double tau_prim = 0.0;
};

struct FockStats {
  long long candidates = 0, quartets = 0, fp32_quartets = 0;
};

struct ScfOptions {
  int max_iter = 100;
  double conv = 1e-10;     // ||P - P_old||_F / 2, as the reference
  int guess = 0;           // 0: P = I (reference), 1: core Hamiltonian, (2: P0 given)
  int diis = 0;            // DIIS subspace size (0 = plain Roothaan, reference)
  double tau = 1e-14;      // Schwarz x density quartet screening threshold
  int mixed = 0;           // 1: incremental Fock builds with FP32 quartets
  double fp32_until = 1e-3;   // all-FP32 builds while ||dP|| is above this
  double tau32 = 1e-7;     // afterwards FP32 only for bounds below this
  int rebuild_every = 6;   // full (non-incremental) build period
  double tau_fp32 = 0.0;   // screening of the FP32 / split builds (0: tau)
  double tau_prim = 0.0;   // primitive-quartet screening of the Fock builds (0: off)
};

struct ScfResult {
  double energy = 0.0, e_nuc = 0.0, delta = 0.0, fock_ms = 0.0, wall_ms = 0.0;
  int iterations = 0, converged = 0;
  long long quartets = 0, fp32_quartets = 0;
};

int scf_run(MolCtx &m, size_t nelec, const ScfOptions &o, ScfResult *res, double *h_P_out,
            const double *h_P0, cudaStream_t st);
int energy_at(MolCtx &m, const double *h_P, double tau, double *E, cudaStream_t st);

// Shell-block maxima of |P| into m.Dsh (nbas x nbas).
void dens_max_device(MolCtx &m, const double *dP, cudaStream_t st);

int mol_create(MolCtx &m, const int *atm, int natm, const int *bas, int nbas, const double *env,
               long long nenv, cudaStream_t st);
void mol_destroy(MolCtx &m, cudaStream_t st);
// G(P) = J - K/2 for a device density dP (n x n, cartesian AOs) into dG
// (added to dG when accumulate).  prec: 0 all FP64, 1 all FP32, 2 FP32 for
// quartets whose Schwarz x density bound is below tau32.  FP32 quartets
// compute the recurrences and the digestion in FP32 and add into the FP64
// J/K accumulators; roots and weights stay FP64.
// rank / nranks: the share of the screened quartets this call digests (the
// candidates whose enumeration index is rank mod nranks); the shares of all
// ranks sum to the full G.
int fock_build(MolCtx &m, const double *dP, double *dG, double tau, cudaStream_t st,
               FockStats *stats, int prec = 0, double tau32 = 0.0, bool accumulate = false,
               int rank = 0, int nranks = 1);
void fill_c2s(double *c);
int int1e_device(int typec, int coord, const int *d_atm, int natm, const int *d_bas, int nbas,
                 const double *d_env, const int *h_bas, double *out, cudaStream_t st,
                 const double *c2s_host);

}  // namespace lrb
