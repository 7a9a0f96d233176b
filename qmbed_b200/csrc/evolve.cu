// Hermitian Krylov exponential action on device vectors.
//
// Reference behaviour (matrixlab-research/QMBED, src/solve/mod.rs):
//   lanczos_projection(_real)             2909-3054
//   projected_exponential_coefficients    3056-3075
//   projected_exponential_action          3077-3129
//   projected_residual_amplitude          3131-3144
//   projected_exponential_error_bound     3146-3195
//   evolve_hermitian_adaptive_grid        3197-3316
//   expm_lanczos                          3432-3454
//   lanczos_spectral_measure              2886-2907
// The recurrence, the real fast path (real operator and exactly real state),
// the a-posteriori error bound and the accept/halve/bisect step control are
// the reference's. Basis vectors live in one column-major FP64 device panel;
// alpha and beta come from fused dot/update kernels with FP64 fixed-tree
// reductions; the tridiagonal eigenproblem runs on the host (implicit QL);
// the projected combination is one pass over the panel.
#include <algorithm>
#include <cmath>

#include "evolve.cuh"

namespace qmbed {

namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr double kPi = 3.14159265358979323846;

// out[i] = sum_b c_b v_b[i] for a real panel (column-major, leading dimension
// n) and complex coefficients c (interleaved); out interleaved complex.
__global__ void combine_real_complex_kernel(const double* __restrict__ panel, uint64_t n, int m,
                                            const double* __restrict__ coeff, double* __restrict__ out) {
  extern __shared__ double c[];
  for (int i = threadIdx.x; i < 2 * m; i += blockDim.x) c[i] = coeff[i];
  __syncthreads();
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double re = 0.0, im = 0.0;
    for (int b = 0; b < m; ++b) {
      const double v = panel[static_cast<uint64_t>(b) * n + i];
      re = fma(c[2 * b], v, re);
      im = fma(c[2 * b + 1], v, im);
    }
    out[2 * i] = re;
    out[2 * i + 1] = im;
  }
}

struct Projection {
  double initial_norm = 0.0;  // norm the basis was normalised with (real part only on the real path)
  double state_norm = 0.0;    // full norm of the projected state
  bool real = false;
  int size = 0;
  double residual_beta = 0.0;
  std::vector<double> eigenvalues;
  std::vector<double> V;  // row-major size x size, eigenvectors as columns
  double vec(int row, int col) const { return V[static_cast<size_t>(row) * size + col]; }
};

// projected_residual_amplitude (src/solve/mod.rs:3131-3144)
double residual_amplitude(const Projection& p, double interval) {
  if (p.size == 0) return 0.0;
  const int last = p.size - 1;
  C64 a(0.0, 0.0);
  for (int e = 0; e < p.size; ++e)
    a += p.initial_norm * p.vec(0, e) * p.vec(last, e) * std::exp(C64(0.0, -interval * p.eigenvalues[e]));
  return std::abs(a);
}

// projected_exponential_error_bound (src/solve/mod.rs:3146-3195)
double error_bound(const Projection& p, double interval, uint64_t n) {
  const double duration = std::fabs(interval);
  if (duration <= kEps || p.size == 0 || static_cast<uint64_t>(p.size) == n || p.residual_beta <= 1.0e-14) return 0.0;
  double lo = INFINITY, hi = -INFINITY;
  for (double v : p.eigenvalues) {
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  const double span = duration * std::max(hi - lo, 0.0);
  const size_t oscillations = static_cast<size_t>(std::min(std::ceil(span / kPi), 60.0));
  size_t intervals = std::min<size_t>(16 + 4 * oscillations, 256);
  if (intervals % 2 != 0) ++intervals;
  const double direction = interval > 0 ? 1.0 : (interval < 0 ? -1.0 : 0.0);
  const double step = duration / static_cast<double>(intervals);
  double integral = 0.0;
  for (size_t i = 0; i <= intervals; ++i) {
    const double w = (i == 0 || i == intervals) ? 1.0 : (i % 2 == 0 ? 2.0 : 4.0);
    integral += w * residual_amplitude(p, direction * step * static_cast<double>(i));
  }
  return 1.25 * p.residual_beta * step * integral / 3.0;
}

class KrylovExp {
 public:
  KrylovExp(const LinearOperatorView& op, BlockOps& ops, size_t krylov)
      : op_(op), ops_(ops), n_(op.dim), m_(static_cast<int>(std::max<uint64_t>(std::min<uint64_t>(krylov, op.dim), 1))) {
    panel_.allocate(static_cast<size_t>(m_) * n_ * 16);
    w_.allocate(std::max<uint64_t>(n_, 1) * 16);
    coeff_.allocate(static_cast<size_t>(2 * m_) * sizeof(double));
  }

  // lanczos_projection(_real) (src/solve/mod.rs:2909-3054) of a device state
  // (interleaved complex FP64). `state_real`: every imaginary part is zero.
  Projection project(const double* state, bool state_real) {
    Projection p;
    p.state_norm = ops_.norm(state, n_, 64, true);
    p.initial_norm = p.state_norm;
    if (p.initial_norm <= kEps) return p;
    p.real = op_.real && state_real;
    const bool cplx = !p.real;
    if (p.real) {
      ops_.import_complex(state, col(0, cplx), n_, 64, false);
      p.initial_norm = ops_.norm(col(0, cplx), n_, 64, false);
      ops_.scale(col(0, cplx), n_, p.initial_norm, 64, false);
    } else {
      ops_.scale_into(state, col(0, cplx), n_, p.initial_norm, 64, true);
    }
    std::vector<double> alphas, betas;
    for (int it = 0; it < m_; ++it) {
      op_.apply(64, cplx, col(it, cplx), w_.get());
      C64 alpha;
      ops_.dots(col(it, cplx), n_, 1, w_.get(), n_, 64, cplx, &alpha);
      if (cplx && std::fabs(alpha.imag()) > 1.0e-10) raise(QMBED_NON_HERMITIAN, "");
      alphas.push_back(alpha.real());
      // w -= beta_{it-1} v_{it-1} + alpha v_it  (one pass over both columns)
      C64 h[2];
      double beta;
      if (it > 0) {
        h[0] = C64(betas[it - 1], 0.0);
        h[1] = C64(alpha.real(), 0.0);
        beta = ops_.subtract(col(it - 1, cplx), n_, 2, h, w_.get(), n_, 64, cplx, true);
      } else {
        h[0] = C64(alpha.real(), 0.0);
        beta = ops_.subtract(col(it, cplx), n_, 1, h, w_.get(), n_, 64, cplx, true);
      }
      p.residual_beta = beta;
      if (it + 1 == m_ || beta <= 1.0e-14) break;
      betas.push_back(beta);
      ops_.scale_into(w_.get(), col(it + 1, cplx), n_, beta, 64, cplx);
    }
    p.size = static_cast<int>(alphas.size());
    tridiagonal_eigen(alphas, std::vector<double>(betas.begin(), betas.begin() + (p.size - 1)), false, p.eigenvalues,
                      p.V);
    return p;
  }

  // projected_exponential_action (src/solve/mod.rs:3056-3129), Hamiltonian
  // form: out = V_m exp(-i t T_m) e_1 |v|, rescaled to the projected norm.
  void action(const Projection& p, double interval, double* out) {
    const cudaStream_t s = ops_.stream();
    if (p.size == 0) {
      QMBED_CUDA(cudaMemsetAsync(out, 0, n_ * 16, s));
      return;
    }
    std::vector<C64> c(p.size, C64(0.0, 0.0));
    for (int e = 0; e < p.size; ++e) {
      const C64 weight = p.initial_norm * p.vec(0, e) * std::exp(C64(0.0, -interval * p.eigenvalues[e]));
      for (int b = 0; b < p.size; ++b) c[b] += p.vec(b, e) * weight;
    }
    if (p.real) {
      QMBED_CUDA(cudaMemcpyAsync(coeff_.get(), c.data(), c.size() * sizeof(C64), cudaMemcpyHostToDevice, s));
      const int blocks = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n_ + 255) / 256, 8ull * ops_.sms())));
      combine_real_complex_kernel<<<blocks, 256, 2 * p.size * sizeof(double), s>>>(panel_.as<double>(), n_, p.size,
                                                                                  coeff_.as<double>(), out);
      QMBED_LAUNCH_CHECK();
      ops_.sync();  // the host coefficients go out of scope
    } else {
      ops_.combine(panel_.get(), n_, p.size, c.data(), 1, out, n_, n_, 64, true);
    }
    const double norm = ops_.norm(out, n_, 64, true);
    if (norm > kEps && std::isfinite(norm)) ops_.scale(out, n_, norm / p.initial_norm, 64, true);
  }

 private:
  void* col(int j, bool cplx) const {
    return static_cast<char*>(panel_.get()) + static_cast<size_t>(j) * n_ * (cplx ? 16 : 8);
  }

  const LinearOperatorView& op_;
  BlockOps& ops_;
  uint64_t n_;
  int m_;
  DeviceBuffer panel_, w_, coeff_;
};

bool host_vector_is_real(const double* v, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i)
    if (v[2 * i + 1] != 0.0) return false;
  return true;
}

}  // namespace

void lanczos_spectral_measure(const LinearOperatorView& op, const double* source, bool source_real, size_t krylov,
                              std::vector<double>& energies, std::vector<double>& weights, BlockOps& ops) {
  if (krylov == 0) raise(QMBED_INVALID_OPTIONS, "spectral Krylov dimension must be positive");
  KrylovExp k(op, ops, krylov);
  const Projection p = k.project(source, source_real);
  energies = p.eigenvalues;
  weights.assign(static_cast<size_t>(p.size), 0.0);
  for (int e = 0; e < p.size; ++e) weights[e] = p.initial_norm * p.initial_norm * p.vec(0, e) * p.vec(0, e);
}

// EvolutionOptions::validate (src/solve/mod.rs:2510-2530)
void validate_evolution(const EvolutionOptions& o) {
  bool ok = !o.times.empty();
  for (size_t i = 0; i < o.times.size(); ++i) {
    ok = ok && std::isfinite(o.times[i]);
    if (i > 0) ok = ok && !(o.times[i - 1] > o.times[i]);
  }
  if (!ok) raise(QMBED_INVALID_OPTIONS, "times must be a nonempty finite nondecreasing grid");
  if (o.krylov_dimension == 0 || !std::isfinite(o.tolerance) || o.tolerance <= 0.0 || o.max_substeps == 0)
    raise(QMBED_INVALID_OPTIONS, "evolution controls must be positive");
}

void evolve(const LinearOperatorView& op, const double* initial, const EvolutionOptions& o, double* states,
            EvolutionDiagnostics& d, BlockOps& ops) {
  validate_evolution(o);
  const uint64_t n = op.dim;
  const cudaStream_t s = ops.stream();
  KrylovExp krylov(op, ops, o.krylov_dimension);
  DeviceBuffer a(std::max<uint64_t>(n, 1) * 16), b(std::max<uint64_t>(n, 1) * 16);
  double* current = a.as<double>();
  double* candidate = b.as<double>();
  QMBED_CUDA(cudaMemcpyAsync(current, initial, n * 16, cudaMemcpyHostToDevice, s));
  bool state_real = host_vector_is_real(initial, n);
  auto emit = [&](size_t t, const double* device) {
    QMBED_CUDA(cudaMemcpyAsync(states + 2 * t * n, device, n * 16, cudaMemcpyDeviceToHost, s));
  };
  double current_time = 0.0;
  size_t output = 0, substeps = 0;
  const double local_tolerance = o.tolerance / static_cast<double>(std::max<size_t>(o.times.size(), 1));
  while (output < o.times.size()) {
    const double target = o.times[output];
    if (std::fabs(target - current_time) <= 16.0 * kEps * std::max(std::fabs(target), 1.0)) {
      emit(output, current);
      current_time = target;
      ++output;
      continue;
    }
    if (substeps >= o.max_substeps) {
      ops.sync();
      raise_nonconvergence(substeps, std::fabs(target - current_time));
    }
    const Projection p = krylov.project(current, state_real);
    d.lanczos_projections += 1;
    d.matrix_vector_products += static_cast<size_t>(p.size);
    if (p.real) {
      d.real_lanczos_projections += 1;
      d.real_matrix_vector_products += static_cast<size_t>(p.size);
    }
    const double threshold = local_tolerance * std::max(p.state_norm, 1.0);
    // the longest accepted prefix of the remaining grid from this projection
    size_t accepted = 0;
    double last_time = current_time;
    for (size_t t = output; t < o.times.size(); ++t) {
      const double interval = o.times[t] - current_time;
      const double error = error_bound(p, interval, n);
      d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
      if (error > threshold) {
        d.rejected_trial_intervals += 1;
        break;
      }
      krylov.action(p, interval, candidate);
      emit(t, candidate);
      ++accepted;
      last_time = o.times[t];
    }
    if (accepted > 0) {
      std::swap(current, candidate);
      current_time = last_time;
      output += accepted;
      ++substeps;
      d.accepted_substeps += 1;
      state_real = false;
      continue;
    }
    const double target_interval = target - current_time;
    const double direction = target_interval > 0 ? 1.0 : (target_interval < 0 ? -1.0 : 0.0);
    const double minimum = 16.0 * kEps * std::max(std::fabs(target), 1.0);
    double rejected = std::fabs(target_interval), magnitude = rejected;
    for (;;) {
      const double error = error_bound(p, direction * magnitude, n);
      d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
      if (error <= threshold || magnitude <= minimum) break;
      d.rejected_trial_intervals += 1;
      rejected = magnitude;
      magnitude *= 0.5;
    }
    if (magnitude > minimum && rejected > magnitude) {
      for (int i = 0; i < 8; ++i) {
        const double trial = 0.5 * (magnitude + rejected);
        const double error = error_bound(p, direction * trial, n);
        d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
        if (error <= threshold) {
          magnitude = trial;
        } else {
          d.rejected_trial_intervals += 1;
          rejected = trial;
        }
      }
    }
    const double interval = direction * magnitude;
    current_time += interval;
    krylov.action(p, interval, candidate);
    std::swap(current, candidate);
    ++substeps;
    d.accepted_substeps += 1;
    state_real = false;
  }
  ops.sync();
}

void expm_lanczos(const LinearOperatorView& op, const double* initial, double time, size_t krylov_dimension,
                  double* out, BlockOps& ops) {
  // LanczosOptions::validate (src/solve/mod.rs:2590-2597) and the finite-time check
  if (krylov_dimension == 0) raise(QMBED_INVALID_OPTIONS, "Lanczos dimension and tolerance must be positive");
  if (!std::isfinite(time)) raise(QMBED_INVALID_OPTIONS, "exponential time must be finite");
  const uint64_t n = op.dim;
  const cudaStream_t s = ops.stream();
  KrylovExp krylov(op, ops, krylov_dimension);
  DeviceBuffer state(std::max<uint64_t>(n, 1) * 16), result(std::max<uint64_t>(n, 1) * 16);
  QMBED_CUDA(cudaMemcpyAsync(state.get(), initial, n * 16, cudaMemcpyHostToDevice, s));
  const Projection p = krylov.project(state.as<double>(), host_vector_is_real(initial, n));
  krylov.action(p, time, result.as<double>());
  QMBED_CUDA(cudaMemcpyAsync(out, result.get(), n * 16, cudaMemcpyDeviceToHost, s));
  ops.sync();
}

void evolve_time_dependent(const TimeDependentOperator& op, const double* initial, double initial_time,
                           const EvolutionOptions& o, double* states, BlockOps& ops) {
  validate_evolution(o);
  if (!std::isfinite(initial_time) || o.times[0] < initial_time)
    raise(QMBED_INVALID_OPTIONS, "initial time must be finite and no later than the first output time");
  if (op.parts.empty()) raise(QMBED_INVALID_OPTIONS, "time-dependent evolution requires a static part");
  const uint64_t n = op.dim;
  const cudaStream_t s = ops.stream();
  const size_t parts = op.parts.size();
  const size_t column = std::max<uint64_t>(n, 1) * 16;
  // columns: rk block [in, k1, k2, k3, k4]; x; part outputs; state; [full, two]; half; error
  DeviceBuffer rk(5 * column), x(column), outputs(parts * column), state(column), pair(2 * column), half(column),
      error(column);
  auto col = [&](const DeviceBuffer& b, size_t j) { return b.as<double>() + 2 * std::max<uint64_t>(n, 1) * j; };
  const uint64_t ld = std::max<uint64_t>(n, 1);
  std::vector<C64> c(parts - 1), weights(parts);
  // derivative -i H(t) x into `out`
  auto derivative = [&](double t, const double* in, double* out) {
    c.assign(parts - 1, C64(std::nan(""), std::nan("")));
    op.coefficients(t, c);
    for (const C64& v : c)
      if (!std::isfinite(v.real()) || !std::isfinite(v.imag()))
        raise(QMBED_INVALID_OPTIONS, "time-dependent coefficient callback did not return " + std::to_string(c.size()) +
                                         " finite values");
    for (size_t j = 0; j < parts; ++j) op.parts[j].apply(64, true, in, col(outputs, j));
    const C64 factor = C64(0.0, -1.0) * op.scale;
    weights[0] = factor;
    for (size_t j = 1; j < parts; ++j) weights[j] = factor * c[j - 1];
    ops.combine(outputs.get(), ld, static_cast<int>(parts), weights.data(), 1, out, ld, n, 64, true);
  };
  auto rk4 = [&](double t, const double* in, double h, double* out) {
    ops.copy(in, col(rk, 0), n * 16);
    derivative(t, col(rk, 0), col(rk, 1));
    const C64 stages[3][4] = {{1.0, 0.5 * h, 0.0, 0.0}, {1.0, 0.0, 0.5 * h, 0.0}, {1.0, 0.0, 0.0, h}};
    const double times[3] = {t + 0.5 * h, t + 0.5 * h, t + h};
    for (int k = 0; k < 3; ++k) {
      ops.combine(rk.get(), ld, k + 2, stages[k], 1, x.get(), ld, n, 64, true);
      derivative(times[k], x.as<double>(), col(rk, k + 2));
    }
    const C64 final_weights[5] = {1.0, h / 6.0, h / 3.0, h / 3.0, h / 6.0};
    ops.combine(rk.get(), ld, 5, final_weights, 1, out, ld, n, 64, true);
  };
  QMBED_CUDA(cudaMemcpyAsync(state.get(), initial, n * 16, cudaMemcpyHostToDevice, s));
  const double requested_norm = ops.norm(state.get(), n, 64, true);
  double previous = initial_time;
  for (size_t output = 0; output < o.times.size(); ++output) {
    const double target = o.times[output];
    const double interval = target - previous;
    if (interval != 0.0) {
      const double direction = interval > 0.0 ? 1.0 : -1.0;
      double h = direction * std::min(std::fabs(interval), 0.1);
      double t = previous;
      size_t steps = 0;
      const double interval_scale = std::max(std::fabs(interval), 1.0);
      while (direction * (target - t) > 16.0 * kEps * std::max(std::fabs(target), 1.0)) {
        if (steps >= o.max_substeps) raise_nonconvergence(steps, std::fabs(target - t));
        if (direction * (t + h - target) > 0.0) h = target - t;
        rk4(t, state.as<double>(), h, col(pair, 0));
        rk4(t, state.as<double>(), 0.5 * h, half.as<double>());
        rk4(t + 0.5 * h, half.as<double>(), 0.5 * h, col(pair, 1));
        const C64 difference[2] = {1.0, -1.0};
        ops.combine(pair.get(), ld, 2, difference, 1, error.get(), ld, n, 64, true);
        const double err = ops.norm(error.get(), n, 64, true);
        const double scale = std::max(ops.norm(col(pair, 1), n, 64, true), 1.0);
        const double threshold = o.tolerance * scale * std::clamp(std::fabs(h) / interval_scale, kEps, 1.0);
        if (err <= threshold || std::fabs(h) <= kEps * std::max(std::fabs(t), 1.0)) {
          ops.copy(col(pair, 1), state.get(), n * 16);
          t += h;
          ++steps;
          h *= err <= kEps ? 2.0 : std::clamp(0.9 * std::pow(threshold / err, 0.2), 1.0, 2.0);
        } else {
          h *= std::clamp(0.9 * std::pow(threshold / err, 0.2), 0.1, 0.8);
        }
      }
    }
    if (requested_norm > kEps) {
      const double norm = ops.norm(state.get(), n, 64, true);
      if (norm <= kEps || !std::isfinite(norm)) raise_nonconvergence(o.max_substeps, norm);
      ops.scale(state.get(), n, norm / requested_norm, 64, true);  // divides by its argument
    }
    QMBED_CUDA(cudaMemcpyAsync(states + 2 * output * n, state.get(), n * 16, cudaMemcpyDeviceToHost, s));
    previous = target;
  }
  ops.sync();
}

}  // namespace qmbed
