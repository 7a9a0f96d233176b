// Explicit sparse operators (CSR) on the GPU.
#include "matrix.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace qmbed {
namespace {

constexpr int kLanesPerRow = 8;  // one row per 8-lane group: rows of QuSpin matrices hold a few dozen entries
constexpr int kThreads = 256;

// y[r] = sum_p A[r, col[p]] x[col[p]]. VAL_CPLX: interleaved complex values;
// VEC_CPLX: interleaved complex vectors. The row loop's trip count is uniform
// across the warp so that every lane reaches the shuffles.
template <bool VAL_CPLX, bool VEC_CPLX>
__global__ void __launch_bounds__(kThreads) csr_apply_kernel(uint64_t n, const uint64_t* __restrict__ row_ptr,
                                                             const uint32_t* __restrict__ cols,
                                                             const double* __restrict__ vals,
                                                             const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x % kLanesPerRow;
  const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kLanesPerRow;
  const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / kLanesPerRow;
  const uint64_t warp_first = group - (threadIdx.x % 32) / kLanesPerRow;  // first group of this warp
  for (uint64_t base = warp_first; base < n; base += groups) {
    const uint64_t r = base + (threadIdx.x % 32) / kLanesPerRow;
    double acc_re = 0.0, acc_im = 0.0;
    if (r < n) {
      const uint64_t end = row_ptr[r + 1];
      for (uint64_t p = row_ptr[r] + lane; p < end; p += kLanesPerRow) {
        const uint32_t c = cols[p];
        if (VAL_CPLX) {
          const double ar = vals[2 * p], ai = vals[2 * p + 1];
          const double xr = x[2 * static_cast<uint64_t>(c)], xi = x[2 * static_cast<uint64_t>(c) + 1];
          acc_re += ar * xr - ai * xi;
          acc_im += ar * xi + ai * xr;
        } else if (VEC_CPLX) {
          const double a = vals[p];
          acc_re += a * x[2 * static_cast<uint64_t>(c)];
          acc_im += a * x[2 * static_cast<uint64_t>(c) + 1];
        } else {
          acc_re += vals[p] * x[c];
        }
      }
    }
    for (int offset = kLanesPerRow / 2; offset > 0; offset /= 2) {
      acc_re += __shfl_xor_sync(0xffffffffu, acc_re, offset);
      if (VEC_CPLX) acc_im += __shfl_xor_sync(0xffffffffu, acc_im, offset);
    }
    if (r < n && lane == 0) {
      if (VEC_CPLX) {
        y[2 * r] = acc_re;
        y[2 * r + 1] = acc_im;
      } else {
        y[r] = acc_re;
      }
    }
  }
}

int sm_count(int device) {
  int sms = 0;
  QMBED_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  return std::max(sms, 1);
}

}  // namespace

CsrMatrix::CsrMatrix(int device, uint64_t n, const std::vector<uint64_t>& rows, const std::vector<uint64_t>& columns,
                     const std::vector<std::complex<double>>& values)
    : device_(device), n_(n) {
  if (rows.size() != columns.size() || rows.size() != values.size())
    raise(QMBED_DIMENSION_MISMATCH, "matrix entry arrays have different lengths");
  if (n > 0xffffffffULL) raise(QMBED_UNSUPPORTED_BACKEND, "explicit matrices are limited to 2^32 rows");
  for (size_t k = 0; k < rows.size(); ++k) {
    if (rows[k] >= n || columns[k] >= n)
      raise(QMBED_DIMENSION_MISMATCH, "matrix entry (" + std::to_string(rows[k]) + ", " +
                                          std::to_string(columns[k]) + ") is outside the matrix shape");
    if (!std::isfinite(values[k].real()) || !std::isfinite(values[k].imag()))
      raise(QMBED_INVALID_OPTIONS, "matrix entries must be finite");
  }
  std::vector<size_t> order(rows.size());
  std::iota(order.begin(), order.end(), size_t{0});
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return rows[a] != rows[b] ? rows[a] < rows[b] : columns[a] < columns[b];
  });
  std::vector<uint64_t> row_ptr(n + 1, 0);
  std::vector<uint32_t> cols;
  std::vector<std::complex<double>> vals;
  cols.reserve(order.size());
  vals.reserve(order.size());
  uint64_t last_row = UINT64_MAX, last_col = UINT64_MAX;
  for (size_t k : order) {
    if (rows[k] == last_row && columns[k] == last_col) {
      vals.back() += values[k];
      continue;
    }
    last_row = rows[k];
    last_col = columns[k];
    cols.push_back(static_cast<uint32_t>(columns[k]));
    vals.push_back(values[k]);
    ++row_ptr[rows[k] + 1];
  }
  for (uint64_t r = 0; r < n; ++r) row_ptr[r + 1] += row_ptr[r];
  nnz_ = cols.size();
  real_ = std::all_of(vals.begin(), vals.end(), [](const std::complex<double>& v) { return v.imag() == 0.0; });

  // shifted_trace_and_one_norm (src/solve/mod.rs:59-100): trace / n as the
  // shift, then the largest column sum of |off-diagonal| + |diagonal - shift|.
  if (n > 0) {
    std::vector<std::complex<double>> diagonal(n, {0.0, 0.0});
    std::vector<double> column_sums(n, 0.0);
    for (uint64_t r = 0; r < n; ++r)
      for (uint64_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
        if (cols[p] == r) diagonal[r] += vals[p];
        else column_sums[cols[p]] += std::abs(vals[p]);
      }
    std::complex<double> trace(0.0, 0.0);
    for (const auto& d : diagonal) trace += d;
    shift_ = trace / static_cast<double>(n);
    for (uint64_t c = 0; c < n; ++c) column_sums[c] += std::abs(diagonal[c] - shift_);
    one_norm_ = *std::max_element(column_sums.begin(), column_sums.end());
  }

  QMBED_CUDA(cudaSetDevice(device_));
  row_ptr_.allocate((n + 1) * sizeof(uint64_t));
  QMBED_CUDA(cudaMemcpy(row_ptr_.get(), row_ptr.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice));
  if (nnz_ > 0) {
    cols_.allocate(nnz_ * sizeof(uint32_t));
    QMBED_CUDA(cudaMemcpy(cols_.get(), cols.data(), nnz_ * sizeof(uint32_t), cudaMemcpyHostToDevice));
    std::vector<double> packed;
    packed.reserve(real_ ? nnz_ : 2 * nnz_);
    for (const auto& v : vals) {
      packed.push_back(v.real());
      if (!real_) packed.push_back(v.imag());
    }
    vals_.allocate(packed.size() * sizeof(double));
    QMBED_CUDA(cudaMemcpy(vals_.get(), packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
}

void CsrMatrix::apply(int precision, bool complex_vectors, const void* x, void* y, cudaStream_t stream) const {
  if (precision != 64) raise(QMBED_UNSUPPORTED_BACKEND, "explicit matrices are applied in FP64");
  if (!real_ && !complex_vectors) raise(QMBED_INVALID_OPTIONS, "a complex matrix needs complex vectors");
  if (n_ == 0) return;
  const size_t row_bytes = (complex_vectors ? 16 : 8) * n_;
  if (nnz_ == 0) {
    QMBED_CUDA(cudaMemsetAsync(y, 0, row_bytes, stream));
    return;
  }
  const uint64_t rows_per_block = kThreads / kLanesPerRow;
  const uint64_t wanted = (n_ + rows_per_block - 1) / rows_per_block;
  const int grid = static_cast<int>(std::min<uint64_t>(wanted, 16ULL * sm_count(device_)));
  const auto* rp = row_ptr_.as<uint64_t>();
  const auto* cp = cols_.as<uint32_t>();
  const auto* vp = vals_.as<double>();
  const auto* xp = static_cast<const double*>(x);
  auto* yp = static_cast<double*>(y);
  if (!real_) csr_apply_kernel<true, true><<<grid, kThreads, 0, stream>>>(n_, rp, cp, vp, xp, yp);
  else if (complex_vectors) csr_apply_kernel<false, true><<<grid, kThreads, 0, stream>>>(n_, rp, cp, vp, xp, yp);
  else csr_apply_kernel<false, false><<<grid, kThreads, 0, stream>>>(n_, rp, cp, vp, xp, yp);
  QMBED_LAUNCH_CHECK();
}

}  // namespace qmbed
