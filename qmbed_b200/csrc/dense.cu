// Complete Hermitian spectra of small sectors.
//
// Reference behaviour (matrixlab-research/QMBED, src/solve/mod.rs):
//   hermitian_eigenpairs_all   558-583 (dense matrix, Hermiticity at 1e-12)
//   eigh / eigh_with_options   585-620 (all pairs, residuals, iterations = 1)
// The reference hands the dense matrix to faer / nalgebra on the host; here
// the matrix is built column by column on the device (column c = H e_c, the
// column-major layout the dense solver wants) and diagonalised by
// cusolverDnZheevd.
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>

#include "dense.cuh"

namespace qmbed {

namespace {

__global__ void unit_vector_kernel(double* __restrict__ x, uint64_t n, uint64_t c) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    x[2 * i] = i == c ? 1.0 : 0.0;
    x[2 * i + 1] = 0.0;
  }
}

// flag |= 1 when |A[r, c] - conj(A[c, r])| > 1e-12 anywhere (A column-major complex).
__global__ void hermitian_flag_kernel(const double2* __restrict__ A, uint64_t n, int* __restrict__ flag) {
  const uint64_t total = n * n;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += stride) {
    const uint64_t r = k % n, c = k / n;
    if (r > c) continue;
    const double2 a = A[c * n + r], b = A[r * n + c];
    const double dr = a.x - b.x, di = a.y + b.y;
    if (hypot(dr, di) > 1.0e-12) atomicOr(flag, 1);
  }
}

// residual partials: out[e] = sum_i |HV[i, e] - lambda_e V[i, e]|^2 (one block per column)
__global__ void residual_columns_kernel(const double2* __restrict__ HV, const double2* __restrict__ V,
                                        const double* __restrict__ lambda, uint64_t n, double* __restrict__ out) {
  const uint64_t e = blockIdx.x;
  double sq = 0.0;
  for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double2 h = HV[e * n + i], v = V[e * n + i];
    const double dr = h.x - lambda[e] * v.x, di = h.y - lambda[e] * v.y;
    sq += dr * dr + di * di;
  }
  __shared__ double red[256];
  red[threadIdx.x] = sq;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[e] = red[0];
}

void check_solver(cusolverStatus_t s, const char* what) {
  if (s != CUSOLVER_STATUS_SUCCESS)
    raise(QMBED_CUDA_ERROR, std::string(what) + " failed with cuSOLVER status " + std::to_string(static_cast<int>(s)));
}

struct SolverHandle {
  cusolverDnHandle_t h = nullptr;
  explicit SolverHandle(cudaStream_t stream) {
    check_solver(cusolverDnCreate(&h), "cusolverDnCreate");
    check_solver(cusolverDnSetStream(h, stream), "cusolverDnSetStream");
  }
  ~SolverHandle() {
    if (h) cusolverDnDestroy(h);
  }
};

}  // namespace

DenseEigensystem dense_eigh(const LinearOperatorView& op, bool want_vectors, BlockOps& ops) {
  const uint64_t n = op.dim;
  DenseEigensystem out;
  if (n == 0) return out;
  if (n > kMaxDenseEigh)
    raise(QMBED_UNSUPPORTED_BACKEND, "dense eigh of more than " + std::to_string(kMaxDenseEigh) +
                                         " states is outside the GPU engine");
  const cudaStream_t stream = ops.stream();
  DeviceBuffer A(n * n * 16), x(n * 16), flag(sizeof(int)), lam(n * 8), info(sizeof(int));
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8ull * ops.sms())));
  for (uint64_t c = 0; c < n; ++c) {
    unit_vector_kernel<<<grid, 256, 0, stream>>>(x.as<double>(), n, c);
    QMBED_LAUNCH_CHECK();
    op.apply(64, true, x.get(), static_cast<char*>(A.get()) + c * n * 16);
  }
  QMBED_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), stream));
  const int hgrid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n * n + 255) / 256, 16ull * ops.sms())));
  hermitian_flag_kernel<<<hgrid, 256, 0, stream>>>(A.as<double2>(), n, flag.as<int>());
  QMBED_LAUNCH_CHECK();
  int nonhermitian = 0;
  QMBED_CUDA(cudaMemcpyAsync(&nonhermitian, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
  ops.sync();
  if (nonhermitian) raise(QMBED_NON_HERMITIAN, "");
  // zheevd overwrites A with the eigenvectors (columns)
  SolverHandle solver(stream);
  const int ni = static_cast<int>(n);
  int lwork = 0;
  check_solver(cusolverDnZheevd_bufferSize(solver.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, ni,
                                           A.as<cuDoubleComplex>(), ni, lam.as<double>(), &lwork),
               "cusolverDnZheevd_bufferSize");
  DeviceBuffer work(static_cast<size_t>(std::max(lwork, 1)) * 16);
  check_solver(cusolverDnZheevd(solver.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, ni,
                                A.as<cuDoubleComplex>(), ni, lam.as<double>(), work.as<cuDoubleComplex>(), lwork,
                                info.as<int>()),
               "cusolverDnZheevd");
  int status = 0;
  QMBED_CUDA(cudaMemcpyAsync(&status, info.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
  out.eigenvalues.resize(n);
  QMBED_CUDA(cudaMemcpyAsync(out.eigenvalues.data(), lam.get(), n * 8, cudaMemcpyDeviceToHost, stream));
  ops.sync();
  if (status != 0) raise_nonconvergence(1, static_cast<double>(status));
  // residuals: the operator applied to each eigenvector, as the reference does
  DeviceBuffer HV(n * n * 16), sq(n * 8);
  for (uint64_t e = 0; e < n; ++e)
    op.apply(64, true, static_cast<char*>(A.get()) + e * n * 16, static_cast<char*>(HV.get()) + e * n * 16);
  residual_columns_kernel<<<static_cast<unsigned>(n), 256, 0, stream>>>(HV.as<double2>(), A.as<double2>(),
                                                                        lam.as<double>(), n, sq.as<double>());
  QMBED_LAUNCH_CHECK();
  out.residuals.resize(n);
  QMBED_CUDA(cudaMemcpyAsync(out.residuals.data(), sq.get(), n * 8, cudaMemcpyDeviceToHost, stream));
  if (want_vectors) {
    out.vectors.resize(n * n);
    QMBED_CUDA(cudaMemcpyAsync(out.vectors.data(), A.get(), n * n * 16, cudaMemcpyDeviceToHost, stream));
  }
  ops.sync();
  for (double& r : out.residuals) r = std::sqrt(std::max(r, 0.0));
  return out;
}

}  // namespace qmbed
