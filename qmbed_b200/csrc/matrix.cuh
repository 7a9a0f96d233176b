// Explicit sparse operators given as matrix entries (the reference's
// MatrixRequest, bindings/capi/src/lib.rs:744-754, built into a stored
// operator by build_operator_model): QuSpin's expm_multiply_parallel and
// other matrix-defined operator models send these.
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace qmbed {

// Square n x n matrix in CSR on one device: row pointers u64, columns u32,
// values FP64 (when every entry is real) or interleaved complex128. Entries
// are sorted by (row, column) and equal positions are summed.
class CsrMatrix {
 public:
  CsrMatrix(int device, uint64_t n, const std::vector<uint64_t>& rows, const std::vector<uint64_t>& columns,
            const std::vector<std::complex<double>>& values);

  uint64_t dim() const { return n_; }
  uint64_t nnz() const { return nnz_; }
  bool is_real() const { return real_; }
  int device() const { return device_; }

  // Trace shift and exact 1-norm of the shifted stored matrix
  // (shifted_trace_and_one_norm, src/solve/mod.rs:59-100).
  std::complex<double> shift() const { return shift_; }
  double one_norm() const { return one_norm_; }

  // y = A x for FP64 vectors: real (only when the matrix is real) or
  // interleaved complex128.
  void apply(int precision, bool complex_vectors, const void* x, void* y, cudaStream_t stream) const;

 private:
  int device_;
  uint64_t n_ = 0, nnz_ = 0;
  bool real_ = true;
  std::complex<double> shift_{0.0, 0.0};
  double one_norm_ = 0.0;
  DeviceBuffer row_ptr_, cols_, vals_;
};

}  // namespace qmbed
