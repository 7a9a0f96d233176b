// Complete Hermitian spectrum of a small sector (the reference's eigh).
#pragma once

#include <vector>

#include "eigsh.cuh"
#include "krylov.cuh"

namespace qmbed {

struct DenseEigensystem {
  std::vector<double> eigenvalues;  // ascending
  std::vector<double> residuals;    // |H v - lambda v|
  std::vector<C64> vectors;         // column e (n values each) belongs to eigenvalues[e]; empty unless requested
};

// eigh / hermitian_eigenpairs_all (src/solve/mod.rs:558-605): the operator's
// dense matrix assembled on the device from its action on unit vectors,
// Hermiticity checked at 1e-12, all eigenpairs by the dense Hermitian
// eigensolver of cuSOLVER, residuals from the device action. Sectors above
// kMaxDenseEigh states are refused.
constexpr uint64_t kMaxDenseEigh = 16384;
DenseEigensystem dense_eigh(const LinearOperatorView& op, bool want_vectors, BlockOps& ops);

}  // namespace qmbed
