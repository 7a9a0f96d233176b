// Selected Hermitian eigenpairs on the GPU: the reference eigsh dispatch
// (dense / expanding Lanczos / thick restart) over device vectors.
#pragma once

#include <complex>
#include <functional>
#include <vector>

#include "krylov.cuh"

namespace qmbed {

enum Target : int { kSmallestAlgebraic = 0, kLargestAlgebraic = 1, kSmallestMagnitude = 2, kLargestMagnitude = 3,
                    kBothEnds = 4, kShift = 5 };

// Reference EigshOptions (src/solve/mod.rs:349-449); krylov_dimension 0 = None.
struct EigshOptions {
  size_t eigenpairs = 1;
  int target = kSmallestAlgebraic;
  double shift = 0.0;
  size_t krylov_dimension = 0;
  double tolerance = 1.0e-10;
  size_t max_iterations = 1000;
  uint64_t seed = 0;
  bool want_vectors = true;  // false: the caller takes eigenvalues only (the filtered solver exports no vectors)
  // Spectral hint (for example from the learned bound network): an interval
  // [hint_lower, hint_upper] believed to hold the spectrum and the gap above
  // the lowest eigenvalue. The filtered solver uses the interval only after a
  // hint_check_steps Lanczos run whose Ritz values it must contain; otherwise
  // it takes its own Lanczos bounds. restart_keep > 0 sets how many Ritz
  // vectors the thick restart keeps per cycle (at least the unconverged
  // wanted ones, at most half the Krylov dimension); 0 keeps the reference's
  // min(needed, m / 2) (src/solve/mod.rs:1799).
  bool hint = false;
  double hint_lower = 0.0, hint_upper = 0.0, hint_gap = 0.0;
  int hint_check_steps = 8;
  size_t restart_keep = 0;
};

enum SolverMode : int {
  kModePlainFP64 = 0,  // the reference algorithms, FP64 vectors
  kModeMixed = 1,      // FP32 vectors and H.v, FP64 recurrences, then FP64 refinement to the tolerance
  kModeFiltered = 2,   // block Chebyshev-filtered subspace iteration, FP32 then FP64 (real operators
                       // with a block action, smallest algebraic); other requests run as kModeMixed
};

struct EigshResult {
  std::vector<double> eigenvalues;
  std::vector<double> residuals;
  size_t iterations = 0;
  size_t reorthogonalization_passes = 0;
  size_t conditional_second_passes = 0;
  bool converged = true;
  bool complex_vectors = false;
  DeviceBuffer vectors;  // FP64, n x k column-major (interleaved complex when complex_vectors)
  // diagnostics
  size_t fp32_iterations = 0;
  size_t fp64_iterations = 0;
  size_t operator_applications = 0;
  int hint_used = 0;               // 1: the hint's interval passed its check and set the filter
  size_t bound_applications = 0;   // operator applications spent on spectral bounds
};

// y = A x on device vectors for the given precision (64/32) and complex flag.
using ApplyFn = std::function<void(int precision, bool cplx, const void* x, void* y)>;

// out = alpha * (S^-1 H S) z + beta * z + gamma * p on row-major n x nb blocks in
// the coordinates z = S^-1 x, S = diag(sqrt(weights)) (SpinOperator::apply_block).
using BlockApplyFn = std::function<void(int precision, int nb, const void* z, const void* p, void* out, double alpha,
                                        double beta, double gamma)>;

struct LinearOperatorView {
  uint64_t dim;
  bool real;  // supports real vectors
  ApplyFn apply;
  BlockApplyFn block_apply = nullptr;  // empty when the operator has no block action
  const uint16_t* weights = nullptr;   // orbit sizes R of the block coordinates; null when every R is 1
};

// Extreme Ritz values of a `steps`-step FP64 Lanczos run without
// reorthogonalisation from the reference deterministic start (seed), with
// the residual norms |beta_m s_m| of their Ritz pairs: Ritz values lie inside
// the spectrum, and an eigenvalue lies within the residual of each.
struct RitzExtremes {
  double min = 0.0, max = 0.0;
  double min_residual = 0.0, max_residual = 0.0;
  int steps = 0;
};
RitzExtremes lanczos_extremes(const LinearOperatorView& op, int steps, uint64_t seed, BlockOps& ops);

// Initial vectors: `n_initial` host vectors of dim complex values,
// interleaved (re, im) doubles, contiguous (may be null when n_initial = 0).
EigshResult eigsh(const LinearOperatorView& op, const EigshOptions& options, const double* initial, int n_initial,
                  int mode, BlockOps& ops);

}  // namespace qmbed
