// Taylor exponential action on the GPU. Reference: ExpmActionPlan::new/apply
// and shifted_trace_and_one_norm (matrixlab-research/QMBED
// src/solve/mod.rs:14-104, 116-248). The theta table and the degree/scaling
// rule (argmin m*s with s = ceil(|c| ||A - mu I||_1 / theta_m)) are the
// reference's published Al-Mohy--Higham constants.
#include <algorithm>
#include <cmath>
#include <limits>

#include "expm.cuh"

namespace qmbed {

namespace {

constexpr std::pair<size_t, double> kTheta[] = {
    {1, 2.29e-16}, {2, 2.58e-8}, {3, 1.39e-5}, {4, 3.40e-4}, {5, 2.40e-3}, {6, 9.07e-3},
    {7, 2.38e-2},  {8, 5.00e-2}, {9, 8.96e-2}, {10, 1.44e-1}, {11, 2.14e-1}, {12, 3.00e-1},
    {13, 4.00e-1}, {14, 5.14e-1}, {15, 6.41e-1}, {16, 7.81e-1}, {17, 9.31e-1}, {18, 1.09},
    {19, 1.26},    {20, 1.44},   {21, 1.62},   {22, 1.82},    {23, 2.01},    {24, 2.22},
    {25, 2.43},    {26, 2.64},   {27, 2.86},   {28, 3.08},    {29, 3.31},    {30, 3.54},
    {35, 4.7},     {40, 6.0},    {45, 7.2},    {50, 8.5},     {55, 9.9},
};

constexpr int kThreads = 256;

// hterm <- scale * (hterm - shift * term); sum += hterm; block maxima of
// |hterm| and |sum| into partials[2 b], partials[2 b + 1].
template <typename T>
__global__ void __launch_bounds__(kThreads) taylor_update_kernel(uint64_t n, T* __restrict__ hterm,
                                                                  const T* __restrict__ term, T* __restrict__ sum,
                                                                  double sr, double si, double mr, double mi,
                                                                  double* __restrict__ partials) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  double m_term = 0.0, m_sum = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double hr = hterm[2 * i], hi = hterm[2 * i + 1];
    const double tr = term[2 * i], ti = term[2 * i + 1];
    const double ur = hr - (mr * tr - mi * ti), ui = hi - (mr * ti + mi * tr);
    const T vr = static_cast<T>(sr * ur - si * ui), vi = static_cast<T>(sr * ui + si * ur);
    hterm[2 * i] = vr;
    hterm[2 * i + 1] = vi;
    const T nr = sum[2 * i] + vr, ni = sum[2 * i + 1] + vi;
    sum[2 * i] = nr;
    sum[2 * i + 1] = ni;
    m_term = fmax(m_term, hypot(static_cast<double>(vr), static_cast<double>(vi)));
    m_sum = fmax(m_sum, hypot(static_cast<double>(nr), static_cast<double>(ni)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    m_term = fmax(m_term, __shfl_xor_sync(0xffffffffu, m_term, o));
    m_sum = fmax(m_sum, __shfl_xor_sync(0xffffffffu, m_sum, o));
  }
  __shared__ double red[kThreads / 32][2];
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = m_term;
    red[threadIdx.x >> 5][1] = m_sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) {
      a = fmax(a, red[w][0]);
      b = fmax(b, red[w][1]);
    }
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) inf_norm_kernel(uint64_t n, const T* __restrict__ v,
                                                             double* __restrict__ partials) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  double m = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    m = fmax(m, hypot(static_cast<double>(v[2 * i]), static_cast<double>(v[2 * i + 1])));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) a = fmax(a, red[w]);
    partials[blockIdx.x] = a;
  }
}

// state <- eta * sum
template <typename T>
__global__ void eta_scale_kernel(uint64_t n, const T* __restrict__ sum, T* __restrict__ state, double er, double ei) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double sr = sum[2 * i], si = sum[2 * i + 1];
    state[2 * i] = static_cast<T>(er * sr - ei * si);
    state[2 * i + 1] = static_cast<T>(er * si + ei * sr);
  }
}

}  // namespace

ExpmPlan make_expm_plan(const SpinOperator& op, C64 coefficient, size_t max_degree, double tolerance,
                        size_t max_substeps) {
  if (!std::isfinite(coefficient.real()) || !std::isfinite(coefficient.imag()) || max_degree == 0 ||
      !std::isfinite(tolerance) || tolerance <= 0.0 || max_substeps == 0)
    raise(QMBED_INVALID_OPTIONS, "invalid exponential coefficient or numerical controls");
  C64 shift;
  double one_norm;
  op.trace_and_one_norm(&shift, &one_norm);
  return make_expm_plan(op.dim(), shift, one_norm, coefficient, max_degree, tolerance, max_substeps);
}

ExpmPlan make_expm_plan(uint64_t dim, C64 shift, double one_norm, C64 coefficient, size_t max_degree,
                        double tolerance, size_t max_substeps) {
  if (!std::isfinite(coefficient.real()) || !std::isfinite(coefficient.imag()) || max_degree == 0 ||
      !std::isfinite(tolerance) || tolerance <= 0.0 || max_substeps == 0)
    raise(QMBED_INVALID_OPTIONS, "invalid exponential coefficient or numerical controls");
  ExpmPlan plan;
  plan.dim = dim;
  plan.coefficient = coefficient;
  plan.tolerance = tolerance;
  plan.shift = shift;
  plan.one_norm = one_norm;
  const double scaled = std::abs(coefficient) * plan.one_norm;
  if (scaled != 0.0) {
    bool found = false;
    size_t best = 0;
    for (auto& [m, theta] : kTheta) {
      if (m > max_degree) continue;
      const size_t s = static_cast<size_t>(std::max(std::ceil(scaled / theta), 1.0));
      if (!found || m * s < best) {
        found = true;
        best = m * s;
        plan.degree = m;
        plan.scaling = s;
      }
    }
    if (!found) raise(QMBED_INVALID_OPTIONS, "Taylor degree is below the minimum supported degree");
  }
  if (plan.scaling > max_substeps) raise_nonconvergence(max_substeps, scaled);
  return plan;
}

size_t expm_apply(const ExpmPlan& plan, const LinearOperatorView& op, void* state, int precision, BlockOps& ops) {
  const uint64_t n = plan.dim;
  if (n == 0) return 0;
  cudaStream_t stream = ops.stream();
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + kThreads - 1) / kThreads,
                                                                             4ULL * ops.sms())));
  DeviceBuffer partials(2 * grid * sizeof(double));
  std::vector<double> host(2 * grid);
  auto read_max = [&](int stride_, int offset) {
    QMBED_CUDA(cudaMemcpyAsync(host.data(), partials.get(), 2 * grid * sizeof(double), cudaMemcpyDeviceToHost, stream));
    QMBED_CUDA(cudaStreamSynchronize(stream));
    double m = 0.0;
    for (int b = 0; b < grid; ++b) m = std::max(m, host[static_cast<size_t>(stride_) * b + offset]);
    return m;
  };
  const size_t bytes = n * 2 * (precision == 64 ? 8 : 4);
  auto inf_norm = [&](const void* v) {
    if (precision == 64) inf_norm_kernel<double><<<grid, kThreads, 0, stream>>>(n, static_cast<const double*>(v), partials.as<double>());
    else inf_norm_kernel<float><<<grid, kThreads, 0, stream>>>(n, static_cast<const float*>(v), partials.as<double>());
    QMBED_LAUNCH_CHECK();
    return read_max(1, 0);
  };
  if (std::abs(plan.coefficient) <= 2.220446049250313e-16 || inf_norm(state) == 0.0) return 0;
  const C64 factor = plan.coefficient / static_cast<double>(plan.scaling);
  const C64 eta = std::exp(factor * plan.shift);
  if (!std::isfinite(eta.real()) || !std::isfinite(eta.imag()))
    raise(QMBED_UNSUPPORTED_BACKEND, "exponential action overflowed its scalar trace shift");
  DeviceBuffer term(bytes), applied(bytes), sum(bytes);
  size_t applications = 0;
  for (size_t s = 0; s < plan.scaling; ++s) {
    ops.copy(state, term.get(), bytes);
    ops.copy(state, sum.get(), bytes);
    double previous = inf_norm(term.get());
    for (size_t order = 1; order <= plan.degree; ++order) {
      op.apply(precision, true, term.get(), applied.get());
      ++applications;
      const C64 scale = factor / static_cast<double>(order);
      if (precision == 64)
        taylor_update_kernel<double><<<grid, kThreads, 0, stream>>>(n, applied.as<double>(), term.as<double>(),
                                                                    sum.as<double>(), scale.real(), scale.imag(),
                                                                    plan.shift.real(), plan.shift.imag(),
                                                                    partials.as<double>());
      else
        taylor_update_kernel<float><<<grid, kThreads, 0, stream>>>(n, applied.as<float>(), term.as<float>(),
                                                                   sum.as<float>(), scale.real(), scale.imag(),
                                                                   plan.shift.real(), plan.shift.imag(),
                                                                   partials.as<double>());
      QMBED_LAUNCH_CHECK();
      std::swap(term, applied);
      QMBED_CUDA(cudaMemcpyAsync(host.data(), partials.get(), 2 * grid * sizeof(double), cudaMemcpyDeviceToHost, stream));
      QMBED_CUDA(cudaStreamSynchronize(stream));
      double term_norm = 0.0, sum_norm = 0.0;
      for (int b = 0; b < grid; ++b) {
        term_norm = std::max(term_norm, host[2 * b]);
        sum_norm = std::max(sum_norm, host[2 * b + 1]);
      }
      if (previous + term_norm <= plan.tolerance * std::max(sum_norm, std::numeric_limits<double>::min())) break;
      previous = term_norm;
    }
    if (precision == 64)
      eta_scale_kernel<double><<<grid, kThreads, 0, stream>>>(n, sum.as<double>(), static_cast<double*>(state),
                                                              eta.real(), eta.imag());
    else
      eta_scale_kernel<float><<<grid, kThreads, 0, stream>>>(n, sum.as<float>(), static_cast<float*>(state),
                                                             eta.real(), eta.imag());
    QMBED_LAUNCH_CHECK();
  }
  QMBED_CUDA(cudaStreamSynchronize(stream));
  return applications;
}

}  // namespace qmbed
