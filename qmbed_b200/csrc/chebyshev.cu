// Chebyshev propagator for the structured flip-chain action.
//
// exp(-i H dt) psi = exp(-i c dt) sum_k (2 - delta_k0) (-i)^k J_k(a dt) T_k(Ht) psi
// with Ht = (H - c) / a, [c - a, c + a] = [e_min, e_max] containing the
// spectrum (Tal-Ezer and Kosloff, J. Chem. Phys. 81, 3967 (1984)). The sum is
// evaluated by the Clenshaw recurrence b_k = c_k psi + 2 Ht b_{k+1} - b_{k+2},
// f = c_0 psi + Ht b_1 - b_2, so no accumulator vector is read or written:
// each step is one fused flip-chain application (two tiled passes) that reads
// b_{k+1}, b_{k+2} and psi and writes b_k over b_{k+2}.
#include <algorithm>
#include <cmath>

#include "chebyshev.cuh"

namespace qmbed {

namespace {

constexpr double kEps = 2.220446049250313e-16;

template <typename T>
__global__ void complex_scale_kernel(uint64_t n, const T* __restrict__ q, T kr, T ki, T* __restrict__ out) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const T re = q[2 * i], im = q[2 * i + 1];
    out[2 * i] = kr * re - ki * im;
    out[2 * i + 1] = kr * im + ki * re;
  }
}

}  // namespace

size_t chebyshev_terms(double x, double tolerance) {
  const double ax = std::fabs(x);
  const double small = tolerance / 8.0;
  size_t k = static_cast<size_t>(std::floor(ax)) + 1;
  for (; k < 1000000; ++k)
    if (std::fabs(std::cyl_bessel_j(static_cast<double>(k), ax)) < small &&
        std::fabs(std::cyl_bessel_j(static_cast<double>(k + 1), ax)) < small)
      break;
  return std::max<size_t>(k, 2);
}

void flip_chain_norm_bounds(const SpinOperator& op, double* e_min, double* e_max) {
  const FlipChain* fc = op.flip_chain();
  if (!fc) raise(QMBED_UNSUPPORTED_BACKEND, "norm bounds need the structured flip-chain action");
  const double b = fc->norm_bound();
  *e_min = -b;
  *e_max = b;
}

namespace {

// The propagation itself: `initial` (interleaved complex128, host or device
// memory per `initial_kind`) evolved over `times`; `output(t, psi, staging)`
// runs after time t with the working-precision state on the device.
template <typename Output>
void chebyshev_run(const SpinOperator& op, const double* initial, cudaMemcpyKind initial_kind,
                   const std::vector<double>& times, double e_min, double e_max, double tolerance, int precision,
                   ChebyshevInfo& info, BlockOps& ops, Output&& output) {
  const FlipChain* fc = op.flip_chain();
  if (!fc)
    raise(QMBED_UNSUPPORTED_BACKEND,
          "the Chebyshev propagator needs the structured flip-chain action (full-space z/x chains, matrix-free)");
  bool ok = !times.empty();
  for (size_t i = 0; i < times.size(); ++i) ok = ok && std::isfinite(times[i]) && (i == 0 || !(times[i - 1] > times[i]));
  if (!ok) raise(QMBED_INVALID_OPTIONS, "times must be a nonempty finite nondecreasing grid");
  if (!(e_max > e_min) || !std::isfinite(e_min) || !std::isfinite(e_max))
    raise(QMBED_INVALID_OPTIONS, "the spectral interval must be finite with e_max > e_min");
  if (!(tolerance > 0.0) || !std::isfinite(tolerance)) raise(QMBED_INVALID_OPTIONS, "tolerance must be positive");
  if (precision != 64 && precision != 32) raise(QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
  QMBED_CUDA(cudaSetDevice(op.basis().device()));
  const uint64_t n = op.dim();
  const size_t es = precision == 64 ? 16 : 8;
  const cudaStream_t s = ops.stream();
  DeviceBuffer staging(n * 16), buf_psi(n * es), buf_a(n * es), buf_b(n * es);
  void* psi = buf_psi.get();
  void* b1 = buf_a.get();
  void* b2 = buf_b.get();
  QMBED_CUDA(cudaMemcpyAsync(staging.get(), initial, n * 16, initial_kind, s));
  ops.convert(staging.get(), 64, psi, precision, 2 * n);
  const double norm0 = ops.norm(psi, n, precision, true);
  const double a = 0.5 * (e_max - e_min), c = 0.5 * (e_max + e_min);
  info.e_min = e_min;
  info.e_max = e_max;
  const int blocks = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8ull * ops.sms())));
  auto scale = [&](const void* q, C64 k, void* out) {
    if (precision == 64)
      complex_scale_kernel<double><<<blocks, 256, 0, s>>>(n, static_cast<const double*>(q), k.real(), k.imag(),
                                                          static_cast<double*>(out));
    else
      complex_scale_kernel<float><<<blocks, 256, 0, s>>>(n, static_cast<const float*>(q), static_cast<float>(k.real()),
                                                         static_cast<float>(k.imag()), static_cast<float*>(out));
    QMBED_LAUNCH_CHECK();
  };
  auto emit = [&](size_t t) {
    output(t, static_cast<const void*>(psi), staging.get());
    const double norm = ops.norm(psi, n, precision, true);
    info.max_norm_drift = std::max(info.max_norm_drift, std::fabs(norm - norm0));
  };
  double previous = 0.0;
  for (size_t t = 0; t < times.size(); ++t) {
    const double dt = times[t] - previous;
    previous = times[t];
    if (std::fabs(dt) <= 16.0 * kEps * std::max(std::fabs(times[t]), 1.0)) {
      emit(t);
      continue;
    }
    const double x = a * dt;
    const double sign = x < 0 ? -1.0 : 1.0;
    const size_t K = chebyshev_terms(x, tolerance);
    std::vector<C64> coef(K);
    const C64 phase = std::exp(C64(0.0, -c * dt));
    C64 minus_i_k(1.0, 0.0);
    double sign_k = 1.0;
    for (size_t k = 0; k < K; ++k) {
      const double jk = sign_k * std::cyl_bessel_j(static_cast<double>(k), std::fabs(x));
      coef[k] = (k == 0 ? 1.0 : 2.0) * minus_i_k * jk * phase;
      minus_i_k *= C64(0.0, -1.0);
      sign_k *= sign;
    }
    // b_{K-1} = c_{K-1} psi; b_K = 0
    scale(psi, coef[K - 1], b1);
    bool b2_valid = false;
    for (size_t k = K - 2; k >= 1; --k) {
      FlipStep step;
      step.alpha = 2.0 / a;
      step.beta = -2.0 * c / a;
      step.gamma = -1.0;
      step.kappa_re = coef[k].real();
      step.kappa_im = coef[k].imag();
      fc->apply(precision, true, b1, b2, b2_valid ? b2 : nullptr, psi, step, s);
      std::swap(b1, b2);
      b2_valid = true;
      ++info.applications;
    }
    // f = c_0 psi + Ht b_1 - b_2, written over b_2 and taken as the new psi
    FlipStep last;
    last.alpha = 1.0 / a;
    last.beta = -c / a;
    last.gamma = -1.0;
    last.kappa_re = coef[0].real();
    last.kappa_im = coef[0].imag();
    fc->apply(precision, true, b1, b2, b2_valid ? b2 : nullptr, psi, last, s);
    ++info.applications;
    std::swap(psi, b2);
    ++info.intervals;
    emit(t);
  }
  ops.sync();
  fc->check_status();  // a multi-pass box wait that timed out
}

}  // namespace

void chebyshev_evolve(const SpinOperator& op, const double* initial, const std::vector<double>& times, double e_min,
                      double e_max, double tolerance, int precision, bool final_only, double* states,
                      ChebyshevInfo& info, BlockOps& ops) {
  const uint64_t n = op.dim();
  const cudaStream_t s = ops.stream();
  chebyshev_run(op, initial, cudaMemcpyHostToDevice, times, e_min, e_max, tolerance, precision, info, ops,
                [&](size_t t, const void* psi, void* staging) {
                  if (final_only && t + 1 != times.size()) return;
                  ops.convert(psi, precision, staging, 64, 2 * n);
                  QMBED_CUDA(cudaMemcpyAsync(states + (final_only ? 0 : 2 * t * n), staging, n * 16,
                                             cudaMemcpyDeviceToHost, s));
                });
}

void chebyshev_evolve_device(const SpinOperator& op, double* state, const std::vector<double>& times, double e_min,
                             double e_max, double tolerance, int precision, ChebyshevInfo& info, BlockOps& ops) {
  const uint64_t n = op.dim();
  chebyshev_run(op, state, cudaMemcpyDeviceToDevice, times, e_min, e_max, tolerance, precision, info, ops,
                [&](size_t t, const void* psi, void*) {
                  if (t + 1 == times.size()) ops.convert(psi, precision, state, 64, 2 * n);
                });
}

}  // namespace qmbed
