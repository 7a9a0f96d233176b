// Hermitian Krylov exponential action exp(-i H t) v on the GPU: Lanczos
// projections without reorthogonalisation and the adaptive time grid of the
// reference evolve.
#pragma once

#include <vector>

#include "eigsh.cuh"

namespace qmbed {

// EvolutionOptions (src/solve/mod.rs:2454-2530).
struct EvolutionOptions {
  std::vector<double> times;
  size_t krylov_dimension = 30;
  double tolerance = 1.0e-10;
  size_t max_substeps = 10000;
};

// EvolutionDiagnostics (src/solve/mod.rs:2546-2555).
struct EvolutionDiagnostics {
  size_t lanczos_projections = 0;
  size_t matrix_vector_products = 0;
  size_t real_lanczos_projections = 0;
  size_t real_matrix_vector_products = 0;
  size_t accepted_substeps = 0;
  size_t rejected_trial_intervals = 0;
  double maximum_estimated_error = 0.0;
};

void validate_evolution(const EvolutionOptions& o);

// evolve with hamiltonian = true (src/solve/mod.rs:3197-3316, 3374-3406).
// `initial` is a host vector of op.dim interleaved complex doubles; the state
// at times[t] is written to states + 2 * t * op.dim (host, interleaved).
void evolve(const LinearOperatorView& op, const double* initial, const EvolutionOptions& o, double* states,
            EvolutionDiagnostics& diagnostics, BlockOps& ops);

// expm_lanczos (src/solve/mod.rs:3432-3454): one projection of dimension
// `krylov`, host vectors in and out (interleaved complex).
void expm_lanczos(const LinearOperatorView& op, const double* initial, double time, size_t krylov, double* out,
                  BlockOps& ops);

// lanczos_spectral_measure (src/solve/mod.rs:2886-2907): Ritz values of the
// unreorthogonalised Lanczos projection of a device vector (interleaved
// complex FP64; `source_real` when every imaginary part is zero) and their
// weights |v|^2 V[0, e]^2.
void lanczos_spectral_measure(const LinearOperatorView& op, const double* source, bool source_real, size_t krylov,
                              std::vector<double>& energies, std::vector<double>& weights, BlockOps& ops);

}  // namespace qmbed
