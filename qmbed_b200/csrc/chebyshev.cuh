// Chebyshev propagator exp(-i H dt) psi for operators with the structured
// flip-chain action, with complex128 or complex64 working vectors.
#pragma once

#include <vector>

#include "krylov.cuh"
#include "operator.cuh"

namespace qmbed {

struct ChebyshevInfo {
  size_t applications = 0;  // H applications over all intervals
  size_t intervals = 0;
  double e_min = 0.0, e_max = 0.0;  // spectral interval used
  double max_norm_drift = 0.0;      // max | ||psi(t)|| - ||psi(0)|| | over the outputs
};

// Terms K of the expansion of exp(-i x y), y in [-1, 1], to `tolerance`:
// the smallest K > x past which |J_k(x)| stays below tolerance / 8.
size_t chebyshev_terms(double x, double tolerance);

// exp(-i H t) initial for each of the nondecreasing `times` (from 0), by one
// Chebyshev expansion per interval on [e_min, e_max] (which must contain the
// spectrum), summed by the Clenshaw recurrence; host vectors (interleaved
// complex FP64) in and out, working precision 64 or 32. With final_only only
// the last state is written (to states[0 .. 2 dim)).
void chebyshev_evolve(const SpinOperator& op, const double* initial, const std::vector<double>& times, double e_min,
                      double e_max, double tolerance, int precision, bool final_only, double* states,
                      ChebyshevInfo& info, BlockOps& ops);

// The same propagation on a device state (interleaved complex128, n
// elements) overwritten with the state at the last time; no host transfers.
void chebyshev_evolve_device(const SpinOperator& op, double* state, const std::vector<double>& times, double e_min,
                             double e_max, double tolerance, int precision, ChebyshevInfo& info, BlockOps& ops);

// Spectral interval guaranteed to contain the spectrum of a flip chain
// (sum of the absolute coefficients on either side of zero).
void flip_chain_norm_bounds(const SpinOperator& op, double* e_min, double* e_max);

}  // namespace qmbed
