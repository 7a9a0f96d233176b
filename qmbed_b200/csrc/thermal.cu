// Full reorthogonalised Lanczos and thermal Lanczos (FTLM / LTLM) on the GPU.
//
// Reference behaviour (matrixlab-research/QMBED, src/solve/mod.rs):
//   LanczosOptions::validate                 2590-2597
//   LanczosIter::next, lanczos_full          2694-2813
//   lanczos_ritz                             2818-2857
//   linear_combination / exponential_action  2636-2671
//   thermal_lanczos_iteration (FTLM = LTLM)  3464-3568
//   thermal observable validation            3596-3644
//   ftlm / ltlm projected contraction        3646-3778
//   project_thermal_observables              3813-3856
// The recurrence is the reference's: three-term step, Gram-Schmidt against
// every stored vector and the current one, repeated once (DGKS) when the norm
// fell to 1/sqrt(2) of its value before. Here the Gram-Schmidt pass is the
// classical (block) form: one pass over the column-major FP64 basis panel
// computes every overlap (alpha among them), a second subtracts them and, in
// the same sweep, reduces the norms before and after reorthogonalisation that
// the DGKS test compares; one host synchronisation per step. The small dense
// work (tridiagonal eigenproblem by implicit QL, Boltzmann sums and
// contractions) is FP64 on the host.
#include <algorithm>
#include <cmath>

#include "thermal.cuh"

namespace qmbed {

namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr double kDgks = 0.70710678118654752440;  // 1/sqrt(2)

int grid_for(uint64_t n, int sms) {
  return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8ull * sms)));
}

// out[i] = sum_b c_b q_b[i] for a real panel and complex coefficients.
__global__ void real_panel_combine_kernel(const double* __restrict__ panel, uint64_t n, int m,
                                          const double* __restrict__ coeff, double* __restrict__ out) {
  extern __shared__ double c[];
  for (int i = threadIdx.x; i < 2 * m; i += blockDim.x) c[i] = coeff[i];
  __syncthreads();
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double re = 0.0, im = 0.0;
    for (int b = 0; b < m; ++b) {
      const double v = panel[static_cast<uint64_t>(b) * n + i];
      re += c[2 * b] * v;
      im += c[2 * b + 1] * v;
    }
    out[2 * i] = re;
    out[2 * i + 1] = im;
  }
}

// re[i] = Re z[i], im[i] = Im z[i]
__global__ void split_complex_kernel(const double* __restrict__ z, double* __restrict__ re, double* __restrict__ im,
                                     uint64_t n) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double2 v = reinterpret_cast<const double2*>(z)[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Rademacher (+-1) entries, or unit phases exp(2 pi i u) with u on a 2^-53
// grid, keyed by (key, i).
__global__ void random_start_kernel(double* __restrict__ out, uint64_t n, uint64_t key, int cplx) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t r = splitmix64(key ^ splitmix64(i));
    if (cplx) {
      double s, c;
      sincospi(2.0 * static_cast<double>(r >> 11) * 0x1.0p-53, &s, &c);
      out[2 * i] = c;
      out[2 * i + 1] = s;
    } else {
      out[i] = (r >> 63) ? -1.0 : 1.0;
    }
  }
}



}  // namespace

void validate_lanczos(size_t krylov, double tolerance) {
  if (krylov == 0 || !std::isfinite(tolerance) || tolerance <= 0.0)
    raise(QMBED_INVALID_OPTIONS, "Lanczos dimension and tolerance must be positive");
}

void lanczos_ritz_device(const LinearOperatorView& op, const double* initial, bool initial_cplx, size_t krylov,
                         double tolerance, LanczosDecomposition& d, BlockOps& ops, bool full_vectors) {
  validate_lanczos(krylov, tolerance);
  const uint64_t n = op.dim;
  if (n == 0) raise(QMBED_DIMENSION_MISMATCH, "Lanczos operator and initial vector do not match");
  QMBED_CUDA(cudaGetDevice(&d.device));
  d.n = n;
  d.real = op.real && !initial_cplx;
  const bool cplx = !d.real;
  const size_t width = cplx ? 16 : 8;
  const uint64_t wanted = std::min<uint64_t>(krylov, n);
  // the overlaps of one step sit in shared memory (16 bytes each)
  if (wanted > 8192) raise(QMBED_UNSUPPORTED_BACKEND, "Krylov dimensions above 8192 are not supported");
  const int capacity = static_cast<int>(wanted);
  const size_t panel_bytes = static_cast<size_t>(capacity) * n * width;
  if (d.basis.bytes() < panel_bytes) d.basis.allocate(panel_bytes);  // kept across repeated runs
  DeviceBuffer w(n * width);
  auto col = [&](int j) { return static_cast<char*>(d.basis.get()) + static_cast<size_t>(j) * n * width; };
  // one Gram-Schmidt pass over q_0 .. q_{m-1}; returns (|w'|^2, |w''|^2, alpha)
  auto pass = [&](int m, double beta, bool three_term, double* before_sq, double* after_sq, C64* alpha) {
    ops.gram_schmidt_pass(d.basis.as<double>(), n, m, beta, three_term, w.as<double>(), cplx, before_sq, after_sq,
                          alpha);
  };

  // normalize (src/solve/mod.rs:694-705) on the caller's vector
  d.initial_norm = ops.norm(initial, n, 64, initial_cplx);
  if (!std::isfinite(d.initial_norm) || d.initial_norm <= kEps) raise_nonconvergence(0, d.initial_norm);
  if (initial_cplx && !cplx) raise(QMBED_INTERNAL_STATE, "complex start on the real path");
  if (cplx && !initial_cplx) {
    DeviceBuffer wide(n * 16);
    ops.widen_real(initial, wide.as<double>(), n);
    ops.scale_into(wide.get(), col(0), n, d.initial_norm, 64, true);
    ops.sync();
  } else {
    ops.scale_into(initial, col(0), n, d.initial_norm, 64, cplx);
  }

  d.diagonal.clear();
  d.off_diagonal.clear();
  d.applications = 0;
  d.second_passes = 0;
  std::vector<double> betas;
  double previous_beta = 0.0;
  for (int index = 0; index < capacity; ++index) {
    op.apply(64, cplx, col(index), w.get());
    ++d.applications;
    // alpha = <q_index, w> is the last overlap of the pass; the pass also
    // yields the norm of the three-term residual (before reorthogonalisation)
    double before_sq, after_sq, unused_sq;
    C64 alpha, again;
    pass(index + 1, previous_beta, true, &before_sq, &after_sq, &alpha);
    if (std::fabs(alpha.imag()) > std::max(tolerance, 1.0e-10)) raise(QMBED_NON_HERMITIAN, "");
    const double before = std::sqrt(std::max(before_sq, 0.0));
    double beta = std::sqrt(std::max(after_sq, 0.0));
    if (before > kEps && beta <= kDgks * before) {  // DGKS: repeat the pass once
      pass(index + 1, 0.0, false, &unused_sq, &after_sq, &again);
      beta = std::sqrt(std::max(after_sq, 0.0));
      ++d.second_passes;
    }
    d.diagonal.push_back(alpha.real());
    betas.push_back(beta);
    if (index + 1 < capacity && beta > tolerance) {
      ops.scale_into(w.get(), col(index + 1), n, beta, 64, cplx);
      previous_beta = beta;
    } else {
      break;
    }
  }
  ops.sync();
  d.size = static_cast<int>(d.diagonal.size());
  d.off_diagonal.assign(betas.begin(), betas.end() - 1);
  d.full_vectors = full_vectors;
  tridiagonal_eigen(d.diagonal, d.off_diagonal, !full_vectors, d.eigenvalues, d.V);
}

void lanczos_ritz(const LinearOperatorView& op, const double* initial, size_t krylov, double tolerance,
                  LanczosDecomposition& d, BlockOps& ops) {
  validate_lanczos(krylov, tolerance);
  const uint64_t n = op.dim;
  if (!initial) raise(QMBED_INVALID_OPTIONS, "Lanczos needs an initial vector");
  bool real = true;
  for (uint64_t i = 0; i < n && real; ++i) real = initial[2 * i + 1] == 0.0;
  DeviceBuffer start(std::max<uint64_t>(n, 1) * 16);
  QMBED_CUDA(cudaMemcpyAsync(start.get(), initial, n * 16, cudaMemcpyHostToDevice, ops.stream()));
  if (op.real && real) {
    DeviceBuffer re(std::max<uint64_t>(n, 1) * 8);
    ops.import_complex(start.as<double>(), re.get(), n, 64, false);
    lanczos_ritz_device(op, re.as<double>(), false, krylov, tolerance, d, ops, true);
  } else {
    lanczos_ritz_device(op, start.as<double>(), true, krylov, tolerance, d, ops, true);
  }
}

ThermalEstimate thermal_estimate(const LanczosDecomposition& d, uint64_t hilbert_dimension,
                                 const std::vector<double>& betas) {
  bool ok = !betas.empty();
  for (double b : betas) ok = ok && std::isfinite(b) && b >= 0.0;
  if (!ok) raise(QMBED_INVALID_OPTIONS, "inverse temperatures must be nonempty, finite, and nonnegative");
  ThermalEstimate t;
  t.krylov_dimension = d.size;
  const double norm_sq = d.initial_norm * d.initial_norm;
  double e_min = INFINITY;
  std::vector<double> weights(static_cast<size_t>(d.size));
  for (int i = 0; i < d.size; ++i) {
    weights[i] = norm_sq * d.vec(0, i) * d.vec(0, i);
    e_min = std::min(e_min, d.eigenvalues[i]);
  }
  for (double beta : betas) {
    double z = 0.0, e = 0.0;
    for (int i = 0; i < d.size; ++i) {
      const double b = weights[i] * std::exp(-beta * (d.eigenvalues[i] - e_min));
      z += b;
      e += b * d.eigenvalues[i];
    }
    if (z <= kEps) raise_nonconvergence(static_cast<size_t>(d.size), z);
    t.log_partition.push_back(std::log(static_cast<double>(hilbert_dimension) / norm_sq) - beta * e_min + std::log(z));
    t.mean_energy.push_back(e / z);
  }
  return t;
}

std::vector<C64> project_observable(const LanczosDecomposition& d, const LinearOperatorView& a, bool ltlm,
                                    BlockOps& ops) {
  if (d.size == 0 || a.dim != d.n)
    raise(QMBED_DIMENSION_MISMATCH, "thermal observables require unique names and matching square shapes");
  const uint64_t n = d.n;
  const int m = d.size;
  std::vector<C64> out(static_cast<size_t>(ltlm ? m : 1) * m);
  const int G = grid_for(n, ops.sms());
  if (!d.real) {
    DeviceBuffer applied(n * 16);
    for (int input = 0; input < (ltlm ? m : 1); ++input) {
      a.apply(64, true, d.column(input), applied.get());
      ops.dots(d.basis.get(), n, m, applied.get(), n, 64, true, out.data() + static_cast<size_t>(input) * m);
    }
  } else if (a.real) {
    DeviceBuffer applied(n * 8);
    for (int input = 0; input < (ltlm ? m : 1); ++input) {
      a.apply(64, false, d.column(input), applied.get());
      ops.dots(d.basis.get(), n, m, applied.get(), n, 64, false, out.data() + static_cast<size_t>(input) * m);
    }
  } else {
    // complex observable on a real basis: widen the input column, split the
    // complex result and take the real and imaginary overlaps separately
    DeviceBuffer wide(n * 16), applied(n * 16), parts(n * 16);
    double* re = parts.as<double>();
    double* im = re + n;
    std::vector<C64> ore(static_cast<size_t>(m)), oim(static_cast<size_t>(m));
    for (int input = 0; input < (ltlm ? m : 1); ++input) {
      ops.widen_real(static_cast<const double*>(d.column(input)), wide.as<double>(), n);
      a.apply(64, true, wide.get(), applied.get());
      split_complex_kernel<<<G, 256, 0, ops.stream()>>>(applied.as<double>(), re, im, n);
      QMBED_LAUNCH_CHECK();
      ops.dots(d.basis.get(), n, m, re, n, 64, false, ore.data());
      ops.dots(d.basis.get(), n, m, im, n, 64, false, oim.data());
      for (int j = 0; j < m; ++j) out[static_cast<size_t>(input) * m + j] = C64(ore[j].real(), oim[j].real());
    }
  }
  return out;
}

std::vector<std::vector<double>> ritz_columns(const LanczosDecomposition& d) {
  std::vector<std::vector<double>> cols(static_cast<size_t>(d.size), std::vector<double>(static_cast<size_t>(d.size)));
  for (int c = 0; c < d.size; ++c)
    for (int r = 0; r < d.size; ++r) cols[c][r] = d.vec(r, c);
  return cols;
}

void thermal_contraction(bool ltlm, const std::vector<double>& eigenvalues,
                         const std::vector<std::vector<double>>& vectors,
                         const std::vector<std::vector<C64>>& projected, const std::vector<double>& betas,
                         std::vector<std::vector<C64>>& values, std::vector<double>& identity) {
  // validate_thermal_ritz_data (3596-3644); names are checked by the caller
  const size_t full = eigenvalues.size();
  bool square = full > 0 && vectors.size() == full;
  for (double e : eigenvalues) square = square && std::isfinite(e);
  for (const auto& v : vectors) {
    square = square && v.size() == full;
    for (double x : v) square = square && std::isfinite(x);
  }
  if (!square) raise(QMBED_DIMENSION_MISMATCH, "thermal Lanczos contraction requires a finite square Ritz eigensystem");
  bool ok = !projected.empty() && !betas.empty();
  for (double b : betas) ok = ok && std::isfinite(b);
  if (!ok) raise(QMBED_INVALID_OPTIONS, "thermal observables and inverse temperatures must be nonempty and valid");
  const size_t expected = ltlm ? full * full : full;
  for (const auto& p : projected) {
    bool good = p.size() == expected;
    for (const C64& x : p) good = good && std::isfinite(x.real()) && std::isfinite(x.imag());
    if (!good) raise(QMBED_DIMENSION_MISMATCH, "thermal observables require unique names and matching finite projections");
  }
  values.assign(projected.size(), {});
  identity.clear();
  if (!ltlm) {
    // coefficient[row] = sum_e V[e][row] V[e][0] exp(-beta E_e)
    for (double beta : betas) {
      std::vector<double> coefficient(full, 0.0);
      for (size_t row = 0; row < full; ++row)
        for (size_t e = 0; e < full; ++e)
          coefficient[row] += vectors[e][row] * vectors[e][0] * std::exp(-beta * eigenvalues[e]);
      identity.push_back(coefficient[0]);
      for (size_t o = 0; o < projected.size(); ++o) {
        C64 s(0.0, 0.0);
        for (size_t row = 0; row < full; ++row) s += projected[o][row] * coefficient[row];
        values[o].push_back(s);
      }
    }
    return;
  }
  // ltlm_effective_dimension: the Ritz states up to the first whose Boltzmann
  // factor at the smallest beta times the largest first component is below eps
  double beta_min = INFINITY, first_max = 0.0;
  for (double b : betas) beta_min = std::min(beta_min, b);
  for (const auto& v : vectors) first_max = std::max(first_max, std::fabs(v[0]));
  size_t m = full;
  for (size_t e = 0; e < full; ++e)
    if (std::exp(-eigenvalues[e] * beta_min) * first_max < kEps) {
      m = e;
      break;
    }
  if (m == 0) raise_nonconvergence(0, 0.0);
  for (double beta : betas) {
    double s = 0.0;
    for (size_t e = 0; e < m; ++e) s += vectors[e][0] * vectors[e][0] * std::exp(-beta * eigenvalues[e]);
    identity.push_back(s);
  }
  for (size_t o = 0; o < projected.size(); ++o) {
    // transformed = V^T M V restricted to the effective states, as two products
    std::vector<C64> left(m * full, C64(0.0, 0.0)), t(m * m, C64(0.0, 0.0));
    for (size_t l = 0; l < m; ++l)
      for (size_t in = 0; in < full; ++in) {
        const double v = vectors[l][in];
        if (v == 0.0) continue;
        const C64* row = projected[o].data() + in * full;
        for (size_t bra = 0; bra < full; ++bra) left[l * full + bra] += v * row[bra];
      }
    for (size_t l = 0; l < m; ++l)
      for (size_t r = 0; r < m; ++r) {
        C64 s(0.0, 0.0);
        for (size_t bra = 0; bra < full; ++bra) s += left[l * full + bra] * vectors[r][bra];
        t[l * m + r] = s;
      }
    for (double beta : betas) {
      std::vector<double> w(m);
      for (size_t e = 0; e < m; ++e) w[e] = vectors[e][0] * std::exp(-0.5 * beta * eigenvalues[e]);
      C64 s(0.0, 0.0);
      for (size_t l = 0; l < m; ++l)
        for (size_t r = 0; r < m; ++r) s += w[l] * t[l * m + r] * w[r];
      values[o].push_back(s);
    }
  }
}

void lanczos_combine(const LanczosDecomposition& d, const std::vector<C64>& c, double* out, BlockOps& ops) {
  if (d.size == 0 || c.size() != static_cast<size_t>(d.size))
    raise(QMBED_DIMENSION_MISMATCH, "basis and coefficient counts must be equal and nonzero");
  const cudaStream_t s = ops.stream();
  if (d.real) {
    DeviceBuffer coeff(c.size() * 16);
    QMBED_CUDA(cudaMemcpyAsync(coeff.get(), c.data(), c.size() * 16, cudaMemcpyHostToDevice, s));
    const int G = grid_for(d.n, ops.sms());
    real_panel_combine_kernel<<<G, 256, 2 * c.size() * sizeof(double), s>>>(d.basis.as<double>(), d.n, d.size,
                                                                             coeff.as<double>(), out);
    QMBED_LAUNCH_CHECK();
    ops.sync();
  } else {
    ops.combine(d.basis.get(), d.n, d.size, c.data(), 1, out, d.n, d.n, 64, true);
    ops.sync();
  }
}

std::vector<C64> exponential_coefficients(const LanczosDecomposition& d, C64 coefficient) {
  if (!std::isfinite(coefficient.real()) || !std::isfinite(coefficient.imag()))
    raise(QMBED_INVALID_OPTIONS, "Lanczos exponential coefficient must be finite");
  if (d.size == 0 || d.V.size() != static_cast<size_t>(d.size) * d.size)
    raise(QMBED_INTERNAL_STATE, "Lanczos Ritz eigensystem is inconsistent");
  std::vector<C64> c(static_cast<size_t>(d.size), C64(0.0, 0.0));
  for (int e = 0; e < d.size; ++e) {
    const C64 weight = d.vec(0, e) * std::exp(coefficient * d.eigenvalues[e]) * d.initial_norm;
    for (int b = 0; b < d.size; ++b) c[b] += weight * d.vec(b, e);
  }
  return c;
}

void ftlm_start_vector(const LinearOperatorView& op, uint64_t seed, int index, double* out, BlockOps& ops) {
  const uint64_t n = op.dim;
  const uint64_t key = seed * 0xD1B54A32D192ED03ull + static_cast<uint64_t>(index) * 0x8CB92BA72F3D8DD7ull + 1;
  random_start_kernel<<<grid_for(n, ops.sms()), 256, 0, ops.stream()>>>(out, n, key, op.real ? 0 : 1);
  QMBED_LAUNCH_CHECK();
}

void ftlm_sample(const LinearOperatorView& op, int vectors, uint64_t seed, size_t krylov, double tolerance,
                 const std::vector<double>& betas, std::vector<double>& log_partition,
                 std::vector<double>& mean_energy, std::vector<int>& lengths, BlockOps& ops) {
  validate_lanczos(krylov, tolerance);
  if (vectors < 1) raise(QMBED_INVALID_OPTIONS, "FTLM needs at least one random vector");
  bool ok = !betas.empty();
  for (double b : betas) ok = ok && std::isfinite(b) && b >= 0.0;
  if (!ok) raise(QMBED_INVALID_OPTIONS, "inverse temperatures must be nonempty, finite, and nonnegative");
  const uint64_t n = op.dim;
  const bool cplx = !op.real;
  DeviceBuffer start(std::max<uint64_t>(n, 1) * (cplx ? 16 : 8));
  log_partition.clear();
  mean_energy.clear();
  lengths.clear();
  LanczosDecomposition d;
  for (int r = 0; r < vectors; ++r) {
    ftlm_start_vector(op, seed, r, start.as<double>(), ops);
    lanczos_ritz_device(op, start.as<double>(), cplx, krylov, tolerance, d, ops, false);
    const ThermalEstimate t = thermal_estimate(d, n, betas);
    log_partition.insert(log_partition.end(), t.log_partition.begin(), t.log_partition.end());
    mean_energy.insert(mean_energy.end(), t.mean_energy.begin(), t.mean_energy.end());
    lengths.push_back(t.krylov_dimension);
  }
}

}  // namespace qmbed
