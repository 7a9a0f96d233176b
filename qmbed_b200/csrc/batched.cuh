// Batched lowest eigenvalues of many independent Hamiltonians H(s, p) =
// sum_k c_k(p) A_k(s): every sector s of a basis family times every point p of
// a parameter scan, in one launch per Lanczos step.
#pragma once

#include <vector>

#include "krylov.cuh"
#include "operator.cuh"

namespace qmbed {

struct ScanResult {
  std::vector<double> eigenvalues;  // [sector][point][eigenpairs]
  std::vector<int> steps;           // [sector][point]: Lanczos steps at convergence (-1: not converged)
  int total_steps = 0;
  size_t applications = 0;          // operator applications summed over all columns
};

// components[s][k] holds A_k of sector s (explicit-value rows, all on sector
// s's basis); coefficients[p * K + k] = c_k(p) (real). Up to 64 points (padded
// to 32 or 64 columns internally), up to 8 components, eigenpairs <= 4.
ScanResult scan_lowest(const std::vector<std::vector<const SpinOperator*>>& components,
                       const std::vector<double>& coefficients, int points, int eigenpairs, double tolerance,
                       int max_steps, uint64_t seed, BlockOps& ops);

}  // namespace qmbed
