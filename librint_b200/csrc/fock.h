// Molecule context and direct Fock build (see fock.cu).
#pragma once
#include <vector>

#include "engine.h"
#include "eri_device.cuh"

namespace lrb {

struct MolCtx {
  int natm = 0, nbas = 0, nao = 0, npairs = 0, npp = 0;
  long long nenv = 0;
  std::vector<int> h_atm, h_bas, h_aooff;
  std::vector<double> h_env;
  std::vector<PairInfo> h_pairs;
  int *atm = nullptr, *bas = nullptr, *aooff = nullptr, *pcls = nullptr;
  double *env = nullptr, *Q = nullptr, *Dsh = nullptr;
  PairInfo *pairs = nullptr;
  PrimPair *pp = nullptr;
};

struct FockStats {
  long long candidates = 0, quartets = 0;
};

struct ScfOptions {
  int max_iter = 100;
  double conv = 1e-10;     // ||P - P_old||_F / 2, as the reference
  int guess = 0;           // 0: P = I (reference), 1: core Hamiltonian
  int diis = 0;            // DIIS subspace size (0 = plain Roothaan, reference)
  double tau = 1e-14;      // Schwarz x density quartet screening threshold
};

struct ScfResult {
  double energy = 0.0, e_nuc = 0.0, delta = 0.0, fock_ms = 0.0, wall_ms = 0.0;
  int iterations = 0, converged = 0;
  long long quartets = 0;
};

int scf_run(MolCtx &m, size_t nelec, const ScfOptions &o, ScfResult *res, double *h_P_out,
            const double *h_P0, cudaStream_t st);
int energy_at(MolCtx &m, const double *h_P, double tau, double *E, cudaStream_t st);

int mol_create(MolCtx &m, const int *atm, int natm, const int *bas, int nbas, const double *env,
               long long nenv, cudaStream_t st);
void mol_destroy(MolCtx &m, cudaStream_t st);
// G(P) = J - K/2 for a device density dP (n x n, cartesian AOs) into dG.
int fock_build(MolCtx &m, const double *dP, double *dG, double tau, cudaStream_t st,
               FockStats *stats);
void fill_c2s(double *c);
int int1e_device(int typec, int coord, const int *d_atm, int natm, const int *d_bas, int nbas,
                 const double *d_env, const int *h_bas, double *out, cudaStream_t st,
                 const double *c2s_host);

}  // namespace lrb
