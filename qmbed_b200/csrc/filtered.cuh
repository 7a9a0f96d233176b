// Block Chebyshev-filtered subspace iteration: the accelerated eigsh for real
// operators with a block action (smallest algebraic eigenpairs).
#pragma once

#include "eigsh.cuh"

namespace qmbed {

// Whether filtered_eigsh handles this request.
bool filtered_applicable(const LinearOperatorView& op, const EigshOptions& o, bool complex_initial);

// Smallest algebraic eigenpairs by Chebyshev-filtered subspace iteration on a
// block of 8 or 16 vectors: FP32 blocks until the residuals reach the FP32
// level, then FP64 blocks to `o.tolerance` under the reference acceptance test
// r <= tol * max(|lambda|, 1). The filter interval comes from a short Lanczos
// run (or verified spectral hints). `staged_initial` holds `n_initial` device
// vectors of interleaved complex FP64 (real parts are used). Throws
// NonConvergence when the iteration limit is reached.
EigshResult filtered_eigsh(const LinearOperatorView& op, const EigshOptions& o, const double* staged_initial,
                           int n_initial, BlockOps& ops);

}  // namespace qmbed
