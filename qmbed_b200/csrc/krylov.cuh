// Dense vector kernels for the Krylov solvers (K5/K6), small FP64 eigensolver
// on the GPU (K7) and device reductions. Every reduction accumulates in FP64
// over a fixed tree, so reruns are bitwise reproducible.
#pragma once

#include <complex>
#include <vector>

#include "common.cuh"

namespace qmbed {

using C64 = std::complex<double>;

// row_ptr = exclusive scan of per-row counts (u32 when the total fits).
// False when QMBED_DENSE=scalar selects the CUDA-core kernels for the dense
// contractions (block Gram, Ritz combinations) instead of the FP64 tensor cores.
bool dense_on_tensor_cores();

uint64_t exclusive_scan_counts(const uint32_t* counts, uint64_t n, DeviceBuffer& row_ptr, bool* is64);
C64 device_sum_complex(const double* interleaved, uint64_t n);
double device_max_shifted_column(const double* diag, const double* offsum, uint64_t n, C64 shift);

// Column-major panels of `n`-element vectors with leading dimension `ld`
// (elements, complex counted once). Precision 64 or 32, real or complex.
class BlockOps {
 public:
  BlockOps(int device, cudaStream_t stream);
  ~BlockOps();
  BlockOps(const BlockOps&) = delete;
  BlockOps& operator=(const BlockOps&) = delete;

  cudaStream_t stream() const { return stream_; }
  int sms() const { return sms_; }

  // out[j] = <A_j, w> (conjugate-linear in A) for j < m; with self_sq, also
  // ||w||^2 from the same pass over w.
  void dots(const void* A, uint64_t ld, int m, const void* w, uint64_t n, int precision, bool cplx, C64* out,
            double* self_sq = nullptr);
  // The same overlaps written to device memory (out: 2 m doubles,
  // interleaved), with no host round trip.
  void dots_device(const void* A, uint64_t ld, int m, const void* w, uint64_t n, int precision, bool cplx,
                   double* out);
  // One classical Gram-Schmidt pass of a Lanczos step over an FP64 panel A
  // (m columns, leading dimension n): h = A^H w, then w -= A h, and from the
  // same sweep |w'|^2 for the three-term residual w' = w - Re(h_{m-1}) A_{m-1}
  // - beta A_{m-2} (when `three_term`) and |w - A h|^2; last_overlap = h_{m-1}.
  // One host synchronisation.
  void gram_schmidt_pass(const double* A, uint64_t n, int m, double beta, bool three_term, double* w, bool cplx,
                         double* before_sq, double* after_sq, C64* last_overlap);
  // w = src - A h with h = A^H src (FP64 panel, m columns, leading dimension
  // n; src may equal w), returning h (m values), |src|^2 and |w|^2 with one
  // host synchronisation.
  void project_out(const double* A, uint64_t n, int m, const double* src, double* w, bool cplx, C64* h,
                   double* src_norm_sq, double* out_norm_sq);
  double norm(const void* w, uint64_t n, int precision, bool cplx);
  // w = src - sum_j h_j A_j (src = w when null); returns ||w|| when `want_norm`.
  double subtract(const void* A, uint64_t ld, int m, const C64* h, void* w, uint64_t n, int precision, bool cplx,
                  bool want_norm, const void* src = nullptr);
  // dst = src / divisor
  void scale_into(const void* src, void* dst, uint64_t n, double divisor, int precision, bool cplx);
  // out_k = sum_j Y[j + m k] A_j for k < K.
  void combine(const void* A, uint64_t ld, int m, const C64* Y, int K, void* out, uint64_t ld_out, uint64_t n,
               int precision, bool cplx);
  void scale(void* w, uint64_t n, double factor, int precision, bool cplx);
  // dst (dst_precision) = src (src_precision), `elements` scalars (complex = 2).
  void convert(const void* src, int src_precision, void* dst, int dst_precision, uint64_t elements);
  void copy(const void* src, void* dst, uint64_t bytes);
  // dst[2i] = src[i], dst[2i+1] = 0 (FP64).
  void widen_real(const double* src, double* dst, uint64_t n);
  // dst (precision, complex or real part only) from an interleaved complex FP64 device vector.
  void import_complex(const double* src, void* dst, uint64_t n, int precision, bool cplx);
  // Reference LCG start vector (deterministic_start, src/solve/mod.rs:729-742),
  // unnormalised, real part only; imaginary parts zero for complex vectors.
  void lcg_start(void* out, uint64_t n, uint64_t seed, int precision, bool cplx);
  // r = y - lambda x; returns ||r||  (FP64 accumulation).
  double residual_norm(const void* y, const void* x, double lambda, uint64_t n, int precision, bool cplx);
  void sync();

  // Device buffer `slot` of at least `bytes`, kept for later calls on this
  // handle (grown, never shrunk) so that repeated solves reuse their blocks,
  // like the reference EigshWorkspace (src/solve/mod.rs:477-526).
  void* workspace(int slot, size_t bytes);
  void release_workspace();

 private:
  void ensure_partials(size_t doubles);
  void ensure_coeffs(size_t bytes);
  int device_;
  cudaStream_t stream_;
  int sms_ = 148;
  DeviceBuffer partials_, results_, coeffs_;
  std::vector<DeviceBuffer> workspace_;
  size_t partials_doubles_ = 0, coeffs_bytes_ = 0;
  double* host_results_ = nullptr;  // pinned
  size_t host_results_doubles_ = 0;
};

// Symmetric tridiagonal eigenproblem on the host by implicit QL with
// Wilkinson shifts: ascending values; V row-major n x n (V[row * n + col],
// column col belongs to values[col]), or only its first row when first_row.
void tridiagonal_eigen(std::vector<double> diag, std::vector<double> off, bool first_row, std::vector<double>& values,
                       std::vector<double>& V);

// Eigen-decomposition of a small dense Hermitian matrix (row-major, n <= 2048)
// by parallel cyclic Jacobi in one CTA. Values are returned unsorted with
// column-major eigenvectors.
void device_hermitian_eigen(int n, const std::vector<C64>& a, std::vector<double>& values, std::vector<C64>& vectors,
                            cudaStream_t stream);

// Ascending eigenpairs of a real symmetric m x m matrix (row-major; the
// symmetric part is used) by the same device Jacobi, with real eigenvectors
// as the columns of V (row-major V[i * m + j]).
void device_symmetric_eigen(int m, const std::vector<double>& a, std::vector<double>& values, std::vector<double>& V,
                            cudaStream_t stream);

}  // namespace qmbed
