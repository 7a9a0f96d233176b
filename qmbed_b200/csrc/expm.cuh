// Exponential action exp(c A) v on the GPU.
#pragma once

#include "eigsh.cuh"
#include "operator.cuh"

namespace qmbed {

// Al-Mohy--Higham truncated Taylor plan (reference ExpmActionPlan,
// src/solve/mod.rs:116-248).
struct ExpmPlan {
  uint64_t dim = 0;
  C64 coefficient{0.0, 0.0};
  C64 shift{0.0, 0.0};
  size_t degree = 0;
  size_t scaling = 1;
  double tolerance = 0.0;
  double one_norm = 0.0;
};

ExpmPlan make_expm_plan(const SpinOperator& op, C64 coefficient, size_t max_degree, double tolerance,
                        size_t max_substeps);

// The same plan from an operator's dimension, trace shift and shifted 1-norm.
ExpmPlan make_expm_plan(uint64_t dim, C64 shift, double one_norm, C64 coefficient, size_t max_degree,
                        double tolerance, size_t max_substeps);

// In-place state <- exp(c A) state for an interleaved complex device vector
// of the given precision (64: complex128, 32: complex64).
// Returns the number of operator applications.
size_t expm_apply(const ExpmPlan& plan, const LinearOperatorView& op, void* state, int precision, BlockOps& ops);

}  // namespace qmbed
