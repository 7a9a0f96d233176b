// Hermitian Krylov exponential action exp(-i H t) v on the GPU: Lanczos
// projections without reorthogonalisation and the adaptive time grid of the
// reference evolve.
#pragma once

#include <functional>
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

// A time-dependent operator H(t) = scale * (A_0 + sum_j c_j(t) A_{j+1}):
// `parts` act on the integrator's stream; `coefficients(t, c)` fills the
// c_j (the reference's apply_coefficients / time_operator_scaled,
// src/interop.rs:477-551).
struct TimeDependentOperator {
  uint64_t dim = 0;
  std::vector<LinearOperatorView> parts;  // static part first, then one per component
  std::function<void(double, std::vector<C64>&)> coefficients;
  C64 scale{1.0, 0.0};
};

// evolve_time_dependent_from (src/solve/mod.rs:4086-4138) with
// hamiltonian = true: adaptive RK4 with step doubling between output times
// (adaptive_time_interval, 3998-4066; rk4_step, 3960-3996; derivative
// -i H(t) x, 3941-3958), the state rescaled to the initial norm at every
// output time. Host vectors as in `evolve`.
void evolve_time_dependent(const TimeDependentOperator& op, const double* initial, double initial_time,
                           const EvolutionOptions& o, double* states, BlockOps& ops);

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
