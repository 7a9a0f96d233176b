// Batched lowest eigenvalues of many independent Hamiltonians H(s, p) =
// sum_k c_k(p) A_k(s): every sector s of a basis family times every point p of
// a parameter scan, in one persistent launch per chunk of Lanczos steps.
#pragma once

#include <vector>

#include "krylov.cuh"
#include "operator.cuh"

namespace qmbed {

struct ScanResult {
  std::vector<double> eigenvalues;  // [sector][point][eigenpairs]
  std::vector<double> residuals;    // [sector][point][eigenpairs]: ||H v - theta v|| / ||v|| in FP64
  std::vector<double> e_max;        // [sector][point]: largest Ritz value at convergence
  std::vector<int> steps;           // [sector][point]: Lanczos steps at convergence (-1: not converged)
  int total_steps = 0;              // first-pass steps of the longest pair
  int pass2_steps = 0;              // steps repeated by the Ritz-vector pass
  size_t applications = 0;          // first-pass operator applications summed over the pairs
  size_t applications_verification = 0;  // second pass and residual applications
  double max_relative_residual = 0.0;    // max over reported pairs of residual / max(|theta|, 1)
  int merged_copies = 0;            // close Ritz values found to be copies of one eigenvector
  int failed_pairs = 0;             // pairs without `eigenpairs` verified values
  bool verified = false;            // every reported pair met residual <= tol max(|theta|, 1)
  bool graph = false;               // first pass replayed from a CUDA graph
  int tuned_blocks_per_sm = 0;      // autotuned resident blocks per SM of the persistent launch
  int tuned_rows_per_warp = 1;      // autotuned rows per warp of its apply phase
  std::vector<double> tuning_ms;    // chunk times of the candidates, most blocks first
  double pass1_seconds = 0.0, seconds = 0.0;
};

// components[s][k] holds A_k of sector s (explicit-value rows, all on sector
// s's basis); coefficients[p * K + k] = c_k(p) (real). Up to 64 points (padded
// to 32 or 64 columns internally), up to 8 components, eigenpairs <= 4.
// Raises NonConvergence unless every pair's reported eigenvalues pass the
// FP64 residual test.
ScanResult scan_lowest(const std::vector<std::vector<const SpinOperator*>>& components,
                       const std::vector<double>& coefficients, int points, int eigenpairs, double tolerance,
                       int max_steps, uint64_t seed, BlockOps& ops);

// Runs the persistent kernel's grid barrier with one block too few on
// `device`; returns the status it ended with (1: the bounded spin timed out).
int scan_barrier_selftest(int device);

}  // namespace qmbed
