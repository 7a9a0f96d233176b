// Full reorthogonalised Lanczos decompositions kept in HBM, and the thermal
// Lanczos estimates built on them: FTLM / LTLM partition functions and
// energies, projected observables, and the Ritz reconstruction of
// exp(c T) e_1 through the stored basis.
#pragma once

#include <vector>

#include "eigsh.cuh"
#include "krylov.cuh"

namespace qmbed {

// lanczos_ritz (src/solve/mod.rs:2818-2857) on the device: `size` orthonormal
// Krylov columns (FP64, real when the operator and the start vector are real,
// interleaved complex otherwise; leading dimension n), the tridiagonal, and its
// ascending eigenpairs (V row-major, column j belongs to eigenvalues[j]; only
// its first row when full_vectors is false).
struct LanczosDecomposition {
  int device = 0;
  uint64_t n = 0;
  bool real = false;
  int size = 0;
  double initial_norm = 0.0;
  DeviceBuffer basis;
  std::vector<double> diagonal, off_diagonal;
  std::vector<double> eigenvalues, V;
  size_t applications = 0;
  int second_passes = 0;     // DGKS second Gram-Schmidt passes
  bool full_vectors = true;  // V holds every row (else the first row only)
  const void* column(int j) const {
    return static_cast<const char*>(basis.get()) + static_cast<size_t>(j) * n * (real ? 8 : 16);
  }
  double vec(int row, int col) const { return V[static_cast<size_t>(row) * size + col]; }
};

// LanczosOptions::validate (src/solve/mod.rs:2590-2597)
void validate_lanczos(size_t krylov, double tolerance);

// lanczos_full over LanczosIter::next (src/solve/mod.rs:2694-2813) from a
// host start vector (interleaved complex, op.dim values). The recurrence
// stops after `krylov` vectors, when beta <= tolerance, or once the Krylov
// space spans the whole sector (dim vectors).
void lanczos_ritz(const LinearOperatorView& op, const double* initial, size_t krylov, double tolerance,
                  LanczosDecomposition& out, BlockOps& ops);

// The same recurrence from a device start vector of `initial_cplx` layout
// (FP64, real or interleaved complex); `full_vectors` false keeps only the
// first row of the Ritz vectors (enough for thermal estimates).
void lanczos_ritz_device(const LinearOperatorView& op, const double* initial, bool initial_cplx, size_t krylov,
                         double tolerance, LanczosDecomposition& out, BlockOps& ops, bool full_vectors);

struct ThermalEstimate {
  std::vector<double> log_partition, mean_energy;
  int krylov_dimension = 0;
};

// thermal_lanczos_iteration (src/solve/mod.rs:3464-3540) on a decomposition of
// a `hilbert_dimension`-dimensional operator.
ThermalEstimate thermal_estimate(const LanczosDecomposition& d, uint64_t hilbert_dimension,
                                 const std::vector<double>& inverse_temperatures);

// project_thermal_observables (src/solve/mod.rs:3813-3856): FTLM keeps
// <q_i|A|q_0> (size values), LTLM <q_j|A|q_i> at i * size + j. `a` runs on
// the stream of `ops`.
std::vector<C64> project_observable(const LanczosDecomposition& d, const LinearOperatorView& a, bool ltlm,
                                    BlockOps& ops);

// thermal_observable_contraction (src/solve/mod.rs:3596-3806). `vectors[c][r]`
// is row r of the eigenvector of eigenvalues[c] (column-oriented, like the
// reference). values[o][b] for observable o and inverse temperature b.
void thermal_contraction(bool ltlm, const std::vector<double>& eigenvalues,
                         const std::vector<std::vector<double>>& vectors,
                         const std::vector<std::vector<C64>>& projected, const std::vector<double>& inverse_temperatures,
                         std::vector<std::vector<C64>>& values, std::vector<double>& identity);

// Column-oriented Ritz vectors of a decomposition.
std::vector<std::vector<double>> ritz_columns(const LanczosDecomposition& d);

// LanczosRitzDecomposition::linear_combination / exponential_action
// (src/solve/mod.rs:2636-2671): out (interleaved complex FP64, device) =
// sum_b coefficients[b] q_b.
void lanczos_combine(const LanczosDecomposition& d, const std::vector<C64>& coefficients, double* out,
                     BlockOps& ops);
std::vector<C64> exponential_coefficients(const LanczosDecomposition& d, C64 coefficient);

// One finite-temperature Lanczos estimate per random start vector: vector r
// has Rademacher entries +-1 (real operators) or unit phases (complex ones)
// drawn from (seed, r), generated on the device. Results are row-major
// [vector][inverse temperature]; krylov[r] is the length of run r.
// Start vector `index` of the sampler into device memory (FP64, real for
// real operators, interleaved complex otherwise).
void ftlm_start_vector(const LinearOperatorView& op, uint64_t seed, int index, double* out, BlockOps& ops);
void ftlm_sample(const LinearOperatorView& op, int vectors, uint64_t seed, size_t krylov, double tolerance,
                 const std::vector<double>& inverse_temperatures, std::vector<double>& log_partition,
                 std::vector<double>& mean_energy, std::vector<int>& krylov_lengths, BlockOps& ops);

}  // namespace qmbed
