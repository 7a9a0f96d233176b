// GPU eigsh drivers.
//
// Reference behaviour (matrixlab-research/QMBED, src/solve/mod.rs):
//   eigsh dispatch                 2335-2350, use_dense_eigsh 364-372
//   expanding_lanczos_eigsh        2242-2328
//   lanczos_eigsh(_real)           1116-1456 (full reorthogonalisation, DGKS 1050-1099)
//   thick_restarted_eigsh(_real)   1651-2167 (orthonormalize_*_with_projection 1520-1642)
//   dense_eigsh                    2198-2240
//   deterministic_start            729-742
// The algorithms, windows, restart rules and acceptance test
// r <= tol * max(|lambda|, 1) are the reference's. Gram-Schmidt passes are
// classical (one multi-dot and one block update over the whole panel) with
// the same DGKS second-pass criterion, instead of one dot/axpy per vector.
// The projected/tridiagonal eigenproblems run on the GPU (device Jacobi).
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

#include "eigsh.cuh"
#include "filtered.cuh"

namespace qmbed {

namespace {

constexpr size_t kGuaranteedDense = 128;
constexpr size_t kAutomaticDense = 256;
constexpr size_t kFullKrylovDenseFallback = 2048;
constexpr size_t kTridiagonalWindow = 96;
constexpr double kEps = 2.220446049250313e-16;
const double kDgks = 1.0 / std::sqrt(2.0);
// FP32 vectors resolve residuals to about 1e-7 of the spectral scale; the mixed
// solver hands over to FP64 refinement below this relative level.
constexpr double kMixedHandover = 2.0e-6;

struct Panel {
  DeviceBuffer buf;
  uint64_t n = 0;
  int cols = 0;
  int prec = 64;
  bool cplx = false;
  size_t es() const { return static_cast<size_t>(prec / 8) * (cplx ? 2 : 1); }
  void alloc(uint64_t n_, int cols_, int prec_, bool cplx_) {
    n = n_;
    cols = cols_;
    prec = prec_;
    cplx = cplx_;
    buf.allocate(std::max<size_t>(1, static_cast<size_t>(n) * cols * es()));
  }
  void* col(int j) const { return static_cast<char*>(buf.get()) + static_cast<size_t>(j) * n * es(); }
};

struct Ctx {
  const LinearOperatorView& op;
  BlockOps& ops;
  int prec;
  bool cplx;
  uint64_t n;
  size_t applications = 0;
  void apply(const void* x, void* y) {
    op.apply(prec, cplx, x, y);
    ++applications;
  }
  size_t es() const { return static_cast<size_t>(prec / 8) * (cplx ? 2 : 1); }
  double norm(const void* w) { return ops.norm(w, n, prec, cplx); }
  void copy(const void* src, void* dst) { ops.copy(src, dst, n * es()); }
  void scale(void* w, double divisor) { ops.scale(w, n, divisor, prec, cplx); }
};

[[noreturn]] void nonconvergence(size_t iterations, double residual) { raise_nonconvergence(iterations, residual); }

// select_indices (src/solve/mod.rs:1002-1036)
std::vector<size_t> select_indices(const std::vector<double>& values, int target, size_t count) {
  std::vector<size_t> idx(values.size());
  std::iota(idx.begin(), idx.end(), 0);
  if (target == kBothEnds) {
    std::sort(idx.begin(), idx.end(), [&](size_t l, size_t r) { return values[l] != values[r] ? values[l] < values[r] : l < r; });
    const size_t lower = count / 2, upper = count - lower;
    std::vector<size_t> selected(idx.begin(), idx.begin() + static_cast<long>(std::min(lower, idx.size())));
    for (size_t i = 0; i < upper && i < idx.size(); ++i) selected.push_back(idx[idx.size() - 1 - i]);
    std::stable_sort(selected.begin(), selected.end(), [&](size_t l, size_t r) { return values[l] < values[r]; });
    return selected;
  }
  auto ordering = [&](double a, double b) {
    switch (target) {
      case kSmallestAlgebraic: return a < b ? -1 : (a > b ? 1 : 0);
      case kLargestAlgebraic: return b < a ? -1 : (b > a ? 1 : 0);
      case kSmallestMagnitude: return std::fabs(a) < std::fabs(b) ? -1 : (std::fabs(a) > std::fabs(b) ? 1 : 0);
      case kLargestMagnitude: return std::fabs(b) < std::fabs(a) ? -1 : (std::fabs(b) > std::fabs(a) ? 1 : 0);
      default: return 0;
    }
  };
  std::sort(idx.begin(), idx.end(), [&](size_t l, size_t r) {
    const int o = ordering(values[l], values[r]);
    return o != 0 ? o < 0 : l < r;
  });
  if (idx.size() > count) idx.resize(count);
  return idx;
}

bool candidate_before(double a, double b, int target) {
  switch (target) {
    case kLargestAlgebraic: return b < a;
    case kSmallestMagnitude: return std::fabs(a) < std::fabs(b);
    case kLargestMagnitude: return std::fabs(b) < std::fabs(a);
    default: return a < b;
  }
}

struct Ortho {
  bool ok;
  size_t passes, second_passes;
  std::vector<C64> projection;
};

// orthonormalize_*_with_projection (src/solve/mod.rs:1520-1642): remove the
// first `ncols` panel columns (locked then basis) from w, a DGKS second pass
// when the norm drops below 1/sqrt(2), then normalise.
// `src` is read, the orthogonalised vector is built in `w` (may equal src),
// and the normalised result is written to `slot` (in place when null).
Ortho orthonormalize(Ctx& c, const Panel& Q, int ncols, int projection_from, const void* src, void* w,
                     void* slot = nullptr) {
  Ortho out{false, 1, 0, {}};
  std::vector<C64> h(std::max(ncols, 1));
  double before, norm;
  const bool fused = c.prec == 64 && Q.n == c.n;
  if (ncols > 0 && fused) {
    // overlaps, subtraction and both norms in two sweeps and one synchronisation
    double before_sq = 0.0, norm_sq = 0.0;
    c.ops.project_out(static_cast<const double*>(Q.col(0)), c.n, ncols, static_cast<const double*>(src),
                      static_cast<double*>(w), c.cplx, h.data(), &before_sq, &norm_sq);
    before = std::sqrt(std::max(before_sq, 0.0));
    norm = std::sqrt(std::max(norm_sq, 0.0));
    out.projection.assign(h.begin() + projection_from, h.begin() + ncols);
  } else if (ncols > 0) {
    double before_sq = 0.0;
    c.ops.dots(Q.col(0), Q.n, ncols, src, c.n, c.prec, c.cplx, h.data(), &before_sq);
    before = std::sqrt(std::max(before_sq, 0.0));
    norm = c.ops.subtract(Q.col(0), Q.n, ncols, h.data(), w, c.n, c.prec, c.cplx, true, src);
    out.projection.assign(h.begin() + projection_from, h.begin() + ncols);
  } else {
    before = c.norm(src);
    norm = before;
    if (src != w) c.copy(src, w);
  }
  const bool second = before > kEps && norm <= kDgks * before;
  if (second) {
    if (ncols > 0 && fused) {
      double unused_sq = 0.0, norm_sq = 0.0;
      c.ops.project_out(static_cast<const double*>(Q.col(0)), c.n, ncols, static_cast<const double*>(w),
                        static_cast<double*>(w), c.cplx, h.data(), &unused_sq, &norm_sq);
      norm = std::sqrt(std::max(norm_sq, 0.0));
    } else if (ncols > 0) {
      c.ops.dots(Q.col(0), Q.n, ncols, w, c.n, c.prec, c.cplx, h.data());
      norm = c.ops.subtract(Q.col(0), Q.n, ncols, h.data(), w, c.n, c.prec, c.cplx, true);
    }
    out.passes = 2;
    out.second_passes = 1;
  }
  if (!std::isfinite(norm) || norm <= 1.0e-14) return out;
  if (slot) c.ops.scale_into(w, slot, c.n, norm, c.prec, c.cplx);
  else c.scale(w, norm);
  out.ok = true;
  return out;
}

void upload_vector(Ctx& c, const std::vector<C64>& host, void* device) {
  const uint64_t n = c.n;
  if (c.prec == 64) {
    std::vector<double> buffer(c.cplx ? 2 * n : n);
    for (uint64_t i = 0; i < n; ++i) {
      if (c.cplx) {
        buffer[2 * i] = host[i].real();
        buffer[2 * i + 1] = host[i].imag();
      } else {
        buffer[i] = host[i].real();
      }
    }
    QMBED_CUDA(cudaMemcpyAsync(device, buffer.data(), buffer.size() * 8, cudaMemcpyHostToDevice, c.ops.stream()));
    c.ops.sync();
  } else {
    std::vector<float> buffer(c.cplx ? 2 * n : n);
    for (uint64_t i = 0; i < n; ++i) {
      if (c.cplx) {
        buffer[2 * i] = static_cast<float>(host[i].real());
        buffer[2 * i + 1] = static_cast<float>(host[i].imag());
      } else {
        buffer[i] = static_cast<float>(host[i].real());
      }
    }
    QMBED_CUDA(cudaMemcpyAsync(device, buffer.data(), buffer.size() * 4, cudaMemcpyHostToDevice, c.ops.stream()));
    c.ops.sync();
  }
}

// deterministic_start (src/solve/mod.rs:729-742) into `out`, normalised.
void start_vector(Ctx& c, uint64_t seed, void* out) {
  c.ops.lcg_start(out, c.n, seed, c.prec, c.cplx);
  const double norm = c.norm(out);
  if (!std::isfinite(norm) || norm <= kEps) nonconvergence(0, norm);
  c.scale(out, norm);
}

struct Candidate {
  double value;
  double residual;
  int slot;  // column in the candidate panel
};

// Stores the result vectors (FP64) from `panel` columns in `order`.
void export_vectors(Ctx& c, const Panel& panel, const std::vector<int>& order, EigshResult& result) {
  result.complex_vectors = c.cplx;
  const size_t es64 = static_cast<size_t>(8) * (c.cplx ? 2 : 1);
  result.vectors.allocate(std::max<size_t>(1, order.size() * c.n * es64));
  for (size_t i = 0; i < order.size(); ++i) {
    void* dst = static_cast<char*>(result.vectors.get()) + i * c.n * es64;
    c.ops.convert(panel.col(order[i]), c.prec, dst, 64, c.n * (c.cplx ? 2 : 1));
  }
  c.ops.sync();
}

// lanczos_eigsh with a fixed window (src/solve/mod.rs:1116-1456).
EigshResult lanczos_window(Ctx& c, const EigshOptions& o, const void* initial_device) {
  const uint64_t n = c.n;
  const size_t requested = o.krylov_dimension ? o.krylov_dimension : std::max<size_t>(8 * o.eigenpairs + 64, 256);
  const size_t krylov = std::min({requested, o.max_iterations, static_cast<size_t>(n)});
  if (krylov <= o.eigenpairs) raise(QMBED_INVALID_OPTIONS, "the effective Krylov dimension must exceed eigenpairs");
  Panel V;
  V.alloc(n, static_cast<int>(krylov), c.prec, c.cplx);
  Panel work;
  work.alloc(n, 1, c.prec, c.cplx);
  void* out = work.col(0);
  if (initial_device) {
    c.copy(initial_device, V.col(0));
    const double norm = c.norm(V.col(0));
    if (!std::isfinite(norm) || norm <= kEps) nonconvergence(0, norm);
    c.scale(V.col(0), norm);
  } else {
    start_vector(c, o.seed, V.col(0));
  }
  std::vector<double> alphas, betas;
  size_t passes = 0, seconds = 0, size = 0;
  for (size_t it = 0; it < krylov; ++it) {
    c.apply(V.col(static_cast<int>(it)), out);
    const int m = static_cast<int>(it + 1);
    double alpha, before, beta;
    if (c.prec == 64) {
      // FP64: alpha, the three-term residual norm and one classical pass over
      // the whole basis come from two sweeps and one host synchronisation;
      // dgks_reorthogonalize (src/solve/mod.rs:1050-1099) repeats the pass
      double before_sq, after_sq;
      C64 a;
      c.ops.gram_schmidt_pass(static_cast<const double*>(V.col(0)), n, m, it > 0 ? betas[it - 1] : 0.0, true,
                              static_cast<double*>(out), c.cplx, &before_sq, &after_sq, &a);
      alpha = a.real();
      before = std::sqrt(std::max(before_sq, 0.0));
      beta = std::sqrt(std::max(after_sq, 0.0));
      passes += 1;
      if (before > kEps && beta <= kDgks * before) {
        c.ops.gram_schmidt_pass(static_cast<const double*>(V.col(0)), n, m, 0.0, false, static_cast<double*>(out),
                                c.cplx, &before_sq, &after_sq, nullptr);
        beta = std::sqrt(std::max(after_sq, 0.0));
        passes += 1;
        seconds += 1;
      }
    } else {
      C64 a;
      c.ops.dots(V.col(static_cast<int>(it)), n, 1, out, n, c.prec, c.cplx, &a);
      alpha = a.real();
      if (it > 0) {
        const C64 h[2] = {C64(betas[it - 1], 0.0), C64(alpha, 0.0)};
        before = c.ops.subtract(V.col(static_cast<int>(it - 1)), n, 2, h, out, n, c.prec, c.cplx, true);
      } else {
        const C64 h[1] = {C64(alpha, 0.0)};
        before = c.ops.subtract(V.col(0), n, 1, h, out, n, c.prec, c.cplx, true);
      }
      // dgks_reorthogonalize over the whole basis (src/solve/mod.rs:1050-1099)
      std::vector<C64> h(m);
      c.ops.dots(V.col(0), n, m, out, n, c.prec, c.cplx, h.data());
      beta = c.ops.subtract(V.col(0), n, m, h.data(), out, n, c.prec, c.cplx, true);
      passes += 1;
      if (before > kEps && beta <= kDgks * before) {
        c.ops.dots(V.col(0), n, m, out, n, c.prec, c.cplx, h.data());
        beta = c.ops.subtract(V.col(0), n, m, h.data(), out, n, c.prec, c.cplx, true);
        passes += 1;
        seconds += 1;
      }
    }
    alphas.push_back(alpha);
    size = it + 1;
    if (it + 1 == krylov || beta <= 1.0e-14) break;
    betas.push_back(beta);
    c.ops.scale_into(out, V.col(static_cast<int>(it + 1)), n, beta, c.prec, c.cplx);
  }
  if (size <= o.eigenpairs) nonconvergence(size, std::numeric_limits<double>::infinity());
  // the tridiagonal eigenproblem (nalgebra SymmetricEigen in the reference) on the host
  std::vector<double> values, vectors;  // vectors row-major: column j belongs to values[j]
  tridiagonal_eigen(std::vector<double>(alphas.begin(), alphas.begin() + static_cast<long>(size)),
                    std::vector<double>(betas.begin(), betas.begin() + static_cast<long>(size - 1)), false, values,
                    vectors);
  const std::vector<size_t> indices = select_indices(values, o.target, o.eigenpairs);
  const int K = static_cast<int>(indices.size());
  std::vector<C64> Y(size * K);
  for (int k = 0; k < K; ++k)
    for (size_t j = 0; j < size; ++j) Y[static_cast<size_t>(k) * size + j] = C64(vectors[j * size + indices[k]], 0.0);
  Panel R;
  R.alloc(n, K, c.prec, c.cplx);
  c.ops.combine(V.col(0), n, static_cast<int>(size), Y.data(), K, R.col(0), n, n, c.prec, c.cplx);
  std::vector<Candidate> candidates;
  for (int k = 0; k < K; ++k) {
    const double norm = c.norm(R.col(k));
    if (!std::isfinite(norm) || norm <= kEps) nonconvergence(0, norm);
    c.scale(R.col(k), norm);
    c.apply(R.col(k), out);
    C64 lam;
    c.ops.dots(R.col(k), n, 1, out, n, c.prec, c.cplx, &lam);
    const double residual = c.ops.residual_norm(out, R.col(k), lam.real(), n, c.prec, c.cplx);
    candidates.push_back({lam.real(), residual, k});
  }
  std::stable_sort(candidates.begin(), candidates.end(),
                   [&](const Candidate& a, const Candidate& b) { return candidate_before(a.value, b.value, o.target); });
  double failure = 0.0;
  for (auto& cand : candidates)
    if (cand.residual > o.tolerance * std::max(std::fabs(cand.value), 1.0)) failure = std::max(failure, cand.residual);
  if (failure > 0.0) nonconvergence(size, failure);
  EigshResult result;
  std::vector<int> order;
  for (auto& cand : candidates) {
    result.eigenvalues.push_back(cand.value);
    result.residuals.push_back(cand.residual);
    order.push_back(cand.slot);
  }
  result.iterations = size;
  result.reorthogonalization_passes = passes;
  result.conditional_second_passes = seconds;
  export_vectors(c, R, order, result);
  return result;
}

// thick_restart_dimension (src/solve/mod.rs:1644-1649)
size_t thick_restart_dimension(const EigshOptions& o, uint64_t n) {
  const size_t window = o.krylov_dimension ? o.krylov_dimension : std::max<size_t>(4 * o.eigenpairs + 24, 32);
  return std::min<size_t>(window, n);
}

// thick_restarted_eigsh_{real,complex} (src/solve/mod.rs:1651-2167).
// `initial` holds n_initial device vectors in the context precision.
EigshResult thick_restart(Ctx& c, const EigshOptions& o, const Panel* initial, int n_initial) {
  const uint64_t n = c.n;
  const int m = static_cast<int>(thick_restart_dimension(o, n));
  const int k = static_cast<int>(o.eigenpairs);
  if (m <= k) raise(QMBED_INVALID_OPTIONS, "the effective Krylov dimension must exceed eigenpairs");
  // Ritz vectors kept per cycle: the reference keeps the unconverged wanted
  // ones (src/solve/mod.rs:1799); a restart_keep hint keeps more of the
  // lowest ones, up to half the Krylov dimension.
  const int wider = static_cast<int>(std::min<size_t>(o.restart_keep, static_cast<size_t>(m)));
  auto keep_for = [&](int active) { return std::max(std::min(std::max(active, wider), m / 2), 1); };
  const int keep_cap = keep_for(k);  // candidates per cycle never exceed this
  Panel Q, W, C, CA, RC, RCA, work;
  Q.alloc(n, k + m, c.prec, c.cplx);  // [locked | basis]
  W.alloc(n, m, c.prec, c.cplx);      // applied actions of the basis
  C.alloc(n, keep_cap, c.prec, c.cplx);   // Ritz candidates of this cycle
  CA.alloc(n, keep_cap, c.prec, c.cplx);  // their actions
  const int retain_cap = std::max(keep_cap, n_initial);
  RC.alloc(n, retain_cap, c.prec, c.cplx);   // vectors retained for the next cycle
  RCA.alloc(n, retain_cap, c.prec, c.cplx);  // their actions
  work.alloc(n, 1, c.prec, c.cplx);
  void* tmp = work.col(0);
  std::vector<double> locked_values, locked_residuals;
  int l = 0;
  int retained = 0;
  bool retained_actions = false;
  for (int i = 0; i < n_initial; ++i) c.copy(initial->col(i), RC.col(i));
  retained = n_initial;
  size_t iterations = 0, passes = 0, seconds = 0;
  double last_residual = std::numeric_limits<double>::infinity();
  uint64_t cycle = 0;
  while (iterations < o.max_iterations && l < k) {
    int b = 0, a = 0;
    const bool reuse = retained > 0 && retained_actions;
    for (int i = 0; i < retained; ++i) {
      void* slot = Q.col(l + b);
      if (reuse) {
        const double norm = c.norm(RC.col(i));
        if (std::isfinite(norm) && norm > 1.0e-14) {
          c.ops.scale_into(RC.col(i), slot, n, norm, c.prec, c.cplx);
          c.ops.scale_into(RCA.col(i), W.col(a), n, norm, c.prec, c.cplx);
          ++b;
          ++a;
        }
      } else {
        Ortho r = orthonormalize(c, Q, l + b, l, RC.col(i), tmp, slot);
        passes += r.passes;
        seconds += r.second_passes;
        if (r.ok) ++b;
      }
      if (b >= m / 2) break;
    }
    retained = 0;
    if (b == 0) {
      start_vector(c, o.seed + cycle * 0x9e3779b9ULL, tmp);
      Ortho r = orthonormalize(c, Q, l, l, tmp, tmp, Q.col(l));
      passes += r.passes;
      seconds += r.second_passes;
      if (r.ok) b = 1;
    }
    if (b == 0) break;
    const int known = a;
    std::vector<std::vector<C64>> projection_columns;
    if (reuse) {
      // The residuals of Ritz pairs from one Krylov space are parallel: the
      // first retained action gives the residual direction and the others
      // leave rounding noise. The reference's absolute 1e-14 test can accept
      // that noise; with the reference's restart size it rarely does, but a
      // widened restart would fill the Krylov slots with noise directions, so
      // it takes the first direction only.
      bool added = false;
      for (int column = 0; column < known; ++column) {
        if (b >= m) break;
        Ortho r = orthonormalize(c, Q, l + b, l, W.col(column), tmp, Q.col(l + b));
        passes += r.passes;
        seconds += r.second_passes;
        projection_columns.emplace_back(r.projection.begin(), r.projection.begin() + column + 1);
        if (r.ok && (wider == 0 || !added)) {
          ++b;
          added = true;
        }
      }
    }
    int cursor = known;
    while (cursor < b && iterations < o.max_iterations && a < m) {
      c.apply(Q.col(l + cursor), W.col(a));
      ++iterations;
      ++a;
      // the raw action stays in W; the orthonormalised direction lands in the next basis slot
      Ortho r = orthonormalize(c, Q, l + b, l, W.col(a - 1), tmp, b < m ? Q.col(l + b) : nullptr);
      passes += r.passes;
      seconds += r.second_passes;
      projection_columns.emplace_back(r.projection.begin(), r.projection.begin() + cursor + 1);
      if (b < m && r.ok) ++b;
      ++cursor;
    }
    b = std::min(b, a);
    if (b == 0) break;
    const int size = b;
    std::vector<C64> P(static_cast<size_t>(size) * size, C64(0.0, 0.0));
    for (int col = 0; col < size && col < static_cast<int>(projection_columns.size()); ++col)
      for (int row = 0; row <= col && row < static_cast<int>(projection_columns[col].size()); ++row) {
        const C64 v = projection_columns[col][row];
        P[static_cast<size_t>(row) * size + col] = v;
        P[static_cast<size_t>(col) * size + row] = std::conj(v);
      }
    std::vector<double> values;
    std::vector<C64> vectors;
    device_hermitian_eigen(size, P, values, vectors, c.ops.stream());
    const int active = k - l;
    const int keep = keep_for(active);
    const std::vector<size_t> indices = select_indices(values, o.target, std::min(keep, size));
    const int K = static_cast<int>(indices.size());
    std::vector<C64> Y(static_cast<size_t>(size) * K);
    for (int kk = 0; kk < K; ++kk)
      for (int j = 0; j < size; ++j) Y[static_cast<size_t>(kk) * size + j] = vectors[indices[kk] * size + j];
    c.ops.combine(Q.col(l), n, size, Y.data(), K, C.col(0), n, n, c.prec, c.cplx);
    c.ops.combine(W.col(0), n, size, Y.data(), K, CA.col(0), n, n, c.prec, c.cplx);
    std::vector<Candidate> candidates;
    for (int kk = 0; kk < K; ++kk) {
      const double norm = c.norm(C.col(kk));
      if (!std::isfinite(norm) || norm <= kEps) nonconvergence(iterations, norm);
      c.scale(C.col(kk), norm);
      c.scale(CA.col(kk), norm);
      C64 lam;
      c.ops.dots(C.col(kk), n, 1, CA.col(kk), n, c.prec, c.cplx, &lam);
      const double residual = c.ops.residual_norm(CA.col(kk), C.col(kk), lam.real(), n, c.prec, c.cplx);
      candidates.push_back({lam.real(), residual, kk});
    }
    std::stable_sort(candidates.begin(), candidates.end(),
                     [&](const Candidate& x, const Candidate& y) { return candidate_before(x.value, y.value, o.target); });
    last_residual = 0.0;
    for (int i = 0; i < static_cast<int>(candidates.size()) && i < active; ++i)
      last_residual = std::max(last_residual, candidates[i].residual);
    // Lock converged pairs, retain the rest (with their actions) in rank order.
    int next = 0;
    for (int rank = 0; rank < static_cast<int>(candidates.size()); ++rank) {
      const Candidate& cand = candidates[rank];
      const bool converged = cand.residual <= o.tolerance * std::max(std::fabs(cand.value), 1.0);
      if (rank < active && converged && l < k) {
        Ortho r = orthonormalize(c, Q, l, 0, C.col(cand.slot), tmp, Q.col(l));
        passes += r.passes;
        seconds += r.second_passes;
        if (r.ok) {
          locked_values.push_back(cand.value);
          locked_residuals.push_back(cand.residual);
          ++l;
        }
      } else if (next < keep) {
        c.copy(C.col(cand.slot), RC.col(next));
        c.copy(CA.col(cand.slot), RCA.col(next));
        ++next;
      }
    }
    retained = next;
    retained_actions = true;
    ++cycle;
  }
  if (l < k) nonconvergence(iterations, last_residual);
  std::vector<int> order(l);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return candidate_before(locked_values[x], locked_values[y], o.target); });
  order.resize(k);
  EigshResult result;
  for (int i : order) {
    result.eigenvalues.push_back(locked_values[i]);
    result.residuals.push_back(locked_residuals[i]);
  }
  result.iterations = iterations;
  result.reorthogonalization_passes = passes;
  result.conditional_second_passes = seconds;
  export_vectors(c, Q, order, result);
  return result;
}

// dense_eigsh (src/solve/mod.rs:2198-2240) with the matrix materialised column
// by column on the GPU and diagonalised by the device Jacobi solver.
EigshResult dense_eigsh(Ctx& c, const EigshOptions& o) {
  const uint64_t n = c.n;
  Panel E, Hc;
  E.alloc(n, static_cast<int>(n), 64, true);  // identity columns
  Hc.alloc(n, static_cast<int>(n), 64, true);
  std::vector<double> host(2 * n * n, 0.0);
  for (uint64_t j = 0; j < n; ++j) host[2 * (j * n + j)] = 1.0;
  // All copies go through the solver stream: the operator runs there, and a
  // legacy-stream copy would not be ordered against it.
  QMBED_CUDA(cudaMemcpyAsync(E.col(0), host.data(), host.size() * 8, cudaMemcpyHostToDevice, c.ops.stream()));
  for (uint64_t j = 0; j < n; ++j) c.op.apply(64, true, E.col(static_cast<int>(j)), Hc.col(static_cast<int>(j)));
  QMBED_CUDA(cudaMemcpyAsync(host.data(), Hc.col(0), host.size() * 8, cudaMemcpyDeviceToHost, c.ops.stream()));
  c.ops.sync();
  std::vector<C64> dense(n * n);  // row-major
  for (uint64_t j = 0; j < n; ++j)
    for (uint64_t i = 0; i < n; ++i) dense[i * n + j] = C64(host[2 * (j * n + i)], host[2 * (j * n + i) + 1]);
  for (uint64_t r = 0; r < n; ++r)
    for (uint64_t col = 0; col < n; ++col)
      if (std::abs(dense[r * n + col] - std::conj(dense[col * n + r])) > 1.0e-12) raise(QMBED_NON_HERMITIAN, "");
  std::vector<double> values;
  std::vector<C64> vectors;
  device_hermitian_eigen(static_cast<int>(n), dense, values, vectors, c.ops.stream());
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return values[a] < values[b]; });
  std::vector<double> sorted(n);
  for (size_t i = 0; i < n; ++i) sorted[i] = values[order[i]];
  const std::vector<size_t> indices = select_indices(sorted, o.target, o.eigenpairs);
  Ctx z{c.op, c.ops, 64, true, n};
  Panel R, out;
  R.alloc(n, static_cast<int>(indices.size()), 64, true);
  out.alloc(n, 1, 64, true);
  EigshResult result;
  std::vector<int> slots;
  for (size_t s = 0; s < indices.size(); ++s) {
    std::vector<C64> v(n);
    for (uint64_t i = 0; i < n; ++i) v[i] = vectors[order[indices[s]] * n + i];
    upload_vector(z, v, R.col(static_cast<int>(s)));
    z.apply(R.col(static_cast<int>(s)), out.col(0));
    C64 vv, vhv;
    z.ops.dots(R.col(static_cast<int>(s)), n, 1, R.col(static_cast<int>(s)), n, 64, true, &vv);
    z.ops.dots(R.col(static_cast<int>(s)), n, 1, out.col(0), n, 64, true, &vhv);
    if (!std::isfinite(vv.real()) || vv.real() <= kEps) nonconvergence(0, std::sqrt(vv.real()));
    const double value = vhv.real() / vv.real();
    const double residual = z.ops.residual_norm(out.col(0), R.col(static_cast<int>(s)), value, n, 64, true);
    result.eigenvalues.push_back(value);
    result.residuals.push_back(residual);
    slots.push_back(static_cast<int>(s));
  }
  result.iterations = 1;
  export_vectors(z, R, slots, result);
  c.applications += z.applications + n;
  return result;
}

// expanding_lanczos_eigsh (src/solve/mod.rs:2242-2328).
EigshResult expanding(Ctx& c, const EigshOptions& o, const Panel* initial, int n_initial) {
  const uint64_t n = c.n;
  if (o.krylov_dimension == 0 && n_initial <= 1) {
    const void* init = n_initial == 1 ? initial->col(0) : nullptr;
    size_t subspace = std::min({std::max<size_t>(8 * o.eigenpairs + 64, 256), static_cast<size_t>(n), o.max_iterations});
    size_t spent = 0;
    for (;;) {
      EigshOptions attempt = o;
      attempt.krylov_dimension = subspace;
      attempt.max_iterations = subspace;
      try {
        EigshResult r = lanczos_window(c, attempt, init);
        r.iterations += spent;
        return r;
      } catch (const Error& e) {
        if (e.code != QMBED_NON_CONVERGENCE) throw;
        spent += e.iterations;
        if (subspace == n && n <= kFullKrylovDenseFallback) {
          EigshResult r = dense_eigsh(c, o);
          r.iterations += spent;
          return r;
        }
        const size_t remaining = o.max_iterations > spent ? o.max_iterations - spent : 0;
        const size_t next = std::min({subspace * 2, static_cast<size_t>(n), remaining});
        if (next <= subspace) nonconvergence(spent, e.residual);
        subspace = next;
      }
    }
  }
  if (o.krylov_dimension >= kTridiagonalWindow && n_initial <= 1)
    return lanczos_window(c, o, n_initial == 1 ? initial->col(0) : nullptr);
  try {
    return thick_restart(c, o, initial, n_initial);
  } catch (const Error& e) {
    if (e.code == QMBED_NON_CONVERGENCE && n <= kFullKrylovDenseFallback && o.max_iterations >= n &&
        (o.krylov_dimension == 0 || o.krylov_dimension == n)) {
      EigshResult r = dense_eigsh(c, o);
      r.iterations += e.iterations;
      return r;
    }
    throw;
  }
}

// EigshOptions::validate (src/solve/mod.rs:425-448)
void validate(const EigshOptions& o, uint64_t n) {
  if (o.eigenpairs == 0 || o.eigenpairs >= n)
    raise(QMBED_INVALID_OPTIONS, "eigenpairs must be positive and smaller than the operator dimension");
  if (!std::isfinite(o.tolerance) || o.tolerance <= 0.0 || o.max_iterations == 0)
    raise(QMBED_INVALID_OPTIONS, "tolerance and max_iterations must be positive");
  if (o.krylov_dimension != 0 && (o.krylov_dimension <= o.eigenpairs || o.krylov_dimension > n))
    raise(QMBED_INVALID_OPTIONS, "krylov_dimension must exceed eigenpairs and not exceed dimension");
  if (o.target == kShift && !std::isfinite(o.shift)) raise(QMBED_INVALID_OPTIONS, "shift must be finite");
  if (o.target == kShift)
    raise(QMBED_UNSUPPORTED_BACKEND, "shift-invert eigsh targets are outside this engine");
  if (o.target < 0 || o.target > kShift) raise(QMBED_INVALID_OPTIONS, "unknown spectrum target");
}

}  // namespace

RitzExtremes lanczos_extremes(const LinearOperatorView& op, int steps, uint64_t seed, BlockOps& ops) {
  const uint64_t n = op.dim;
  if (steps < 1) raise(QMBED_INVALID_OPTIONS, "Lanczos steps must be positive");
  const bool cplx = !op.real;
  const size_t es = cplx ? 16 : 8;
  const int m = static_cast<int>(std::min<uint64_t>(static_cast<uint64_t>(steps), n));
  DeviceBuffer a(n * es), b(n * es), w(n * es);
  void* prev = a.get();
  void* cur = b.get();
  ops.lcg_start(cur, n, seed, 64, cplx);
  const double n0 = ops.norm(cur, n, 64, cplx);
  if (!(n0 > kEps)) nonconvergence(0, n0);
  ops.scale(cur, n, n0, 64, cplx);
  std::vector<double> alpha, beta;
  for (int j = 0; j < m; ++j) {
    op.apply(64, cplx, cur, w.get());
    C64 h;
    ops.dots(cur, n, 1, w.get(), n, 64, cplx, &h);
    const C64 ha(h.real(), 0.0);
    double norm = ops.subtract(cur, n, 1, &ha, w.get(), n, 64, cplx, j == 0);
    if (j > 0) {
      const C64 hb(beta.back(), 0.0);
      norm = ops.subtract(prev, n, 1, &hb, w.get(), n, 64, cplx, true);
    }
    alpha.push_back(h.real());
    beta.push_back(norm);
    if (!(norm > 1.0e-12 * std::max(1.0, std::fabs(h.real())))) break;
    // the next vector overwrites the previous one
    ops.scale_into(w.get(), prev, n, norm, 64, cplx);
    std::swap(prev, cur);
  }
  const int size = static_cast<int>(alpha.size());
  std::vector<double> vals, vecs;
  tridiagonal_eigen(alpha, std::vector<double>(beta.begin(), beta.begin() + (size - 1)), false, vals, vecs);
  RitzExtremes r;
  r.steps = size;
  r.min = vals.front();
  r.max = vals.back();
  r.min_residual = std::fabs(beta.back() * vecs[static_cast<size_t>(size - 1) * size + 0]);
  r.max_residual = std::fabs(beta.back() * vecs[static_cast<size_t>(size - 1) * size + (size - 1)]);
  return r;
}

EigshResult eigsh(const LinearOperatorView& op, const EigshOptions& options, const double* initial, int n_initial,
                  int mode, BlockOps& ops) {
  const uint64_t n = op.dim;
  validate(options, n);
  if (mode != kModePlainFP64 && mode != kModeMixed && mode != kModeFiltered)
    raise(QMBED_INVALID_OPTIONS, "unknown solver mode");
  // validate_eigsh_initial (src/solve/mod.rs:660-688)
  bool complex_initial = false;
  for (int k = 0; k < n_initial; ++k) {
    const double* v = initial + 2 * static_cast<size_t>(k) * n;
    double sq = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
      const double re = v[2 * i], im = v[2 * i + 1];
      if (!std::isfinite(re) || !std::isfinite(im))
        raise(QMBED_INVALID_OPTIONS, "eigsh initial vector must contain only finite values");
      if (std::fabs(im) > 1.0e-14) complex_initial = true;
      sq += re * re + im * im;
    }
    if (!std::isfinite(std::sqrt(sq)) || std::sqrt(sq) <= kEps)
      raise(QMBED_INVALID_OPTIONS, "eigsh initial vector must have nonzero finite norm");
  }
  const bool cplx = !op.real || complex_initial;
  // One upload of the caller's vectors; precision/real-part conversion on the device.
  DeviceBuffer staged;
  if (n_initial > 0) {
    staged.allocate(static_cast<size_t>(n_initial) * n * 16);
    QMBED_CUDA(cudaMemcpyAsync(staged.get(), initial, static_cast<size_t>(n_initial) * n * 16,
                               cudaMemcpyHostToDevice, ops.stream()));
  }
  Ctx c64{op, ops, 64, cplx, n};
  if (n <= kGuaranteedDense || (n <= kAutomaticDense && options.krylov_dimension == 0)) {
    EigshResult r = dense_eigsh(c64, options);
    r.operator_applications = c64.applications;
    r.fp64_iterations = r.iterations;
    return r;
  }
  auto upload_initial = [&](Ctx& c, Panel& panel) {
    if (n_initial == 0) return 0;
    panel.alloc(n, n_initial, c.prec, c.cplx);
    for (int i = 0; i < n_initial; ++i)
      c.ops.import_complex(staged.as<double>() + 2 * static_cast<size_t>(i) * n, panel.col(i), n, c.prec, c.cplx);
    return n_initial;
  };
  if (mode == kModeFiltered && filtered_applicable(op, options, complex_initial)) {
    try {
      return filtered_eigsh(op, options, staged.as<double>(), n_initial, ops);
    } catch (const Error& e) {
      if (e.code != QMBED_NON_CONVERGENCE) throw;  // otherwise the mixed Lanczos path below decides
    }
  }
  if (mode == kModePlainFP64) {
    Panel init;
    const int n_init = upload_initial(c64, init);
    EigshResult r = expanding(c64, options, &init, n_init);
    r.operator_applications = c64.applications;
    r.fp64_iterations = r.iterations;
    return r;
  }
  // Mixed precision: FP32 vectors and H.v to the handover tolerance, then the
  // FP64 thick restart seeded with the FP32 Ritz vectors to the requested one.
  Ctx c32{op, ops, 32, cplx, n};
  EigshOptions first = options;
  first.tolerance = std::max(options.tolerance, kMixedHandover);
  // Both phases keep the reference's restart size: the FP32 phase's FP32
  // actions leave rounding noise in the residual directions, and the FP64
  // phase starts from converged FP32 Ritz vectors, where a wider restart was
  // measured to add steps (437 -> 525 at 28 sites); the hint's restart size
  // serves the plain FP64 thick restart.
  first.restart_keep = 0;
  Panel init32;
  const int n_init32 = upload_initial(c32, init32);
  EigshResult phase1;
  try {
    phase1 = expanding(c32, first, &init32, n_init32);
  } catch (const Error& e) {
    if (e.code != QMBED_NON_CONVERGENCE) throw;
    // the FP64 reference algorithms as the fallback, with the spent work counted
    Panel init;
    const int n_init = upload_initial(c64, init);
    EigshOptions rest = options;
    rest.max_iterations = options.max_iterations > e.iterations ? options.max_iterations - e.iterations : 1;
    EigshResult r = expanding(c64, rest, &init, n_init);
    r.fp32_iterations = e.iterations;
    r.fp64_iterations = r.iterations;
    r.iterations += e.iterations;
    r.operator_applications = c32.applications + c64.applications;
    return r;
  }
  const int k = static_cast<int>(phase1.eigenvalues.size());
  // FP64 refinement of the FP32 Ritz vectors. Real operators with a block
  // action refine them as one block through the filtered solver's FP64 phase
  // (its start subspace already holds the wanted pairs to the FP32 level, so it
  // skips its FP32 phase and filters in FP64 to the tolerance); every other
  // operator, or a refinement that does not converge, takes the FP64 thick
  // restart seeded with them.
  if (!cplx && filtered_applicable(op, options, false)) {
    DeviceBuffer wide(static_cast<size_t>(k) * n * 16);
    ops.widen_real(phase1.vectors.as<double>(), wide.as<double>(), static_cast<uint64_t>(k) * n);
    try {
      EigshResult r = filtered_eigsh(op, options, wide.as<double>(), k, ops);
      r.fp32_iterations = phase1.iterations;
      r.fp64_iterations = r.iterations;
      r.iterations += phase1.iterations;
      r.reorthogonalization_passes += phase1.reorthogonalization_passes;
      r.conditional_second_passes += phase1.conditional_second_passes;
      r.operator_applications += c32.applications;
      return r;
    } catch (const Error& e) {
      if (e.code != QMBED_NON_CONVERGENCE) throw;
    }
  }
  Panel seed;
  seed.alloc(n, k, 64, cplx);
  ops.copy(phase1.vectors.get(), seed.col(0), static_cast<size_t>(k) * n * (cplx ? 16 : 8));
  EigshOptions second = options;
  second.restart_keep = 0;
  if (second.krylov_dimension == 0 || second.krylov_dimension >= kTridiagonalWindow)
    second.krylov_dimension = std::min<size_t>(std::max<size_t>(4 * options.eigenpairs + 24, 32), n);
  if (second.krylov_dimension <= second.eigenpairs) second.krylov_dimension = std::min<size_t>(second.eigenpairs + 1, n);
  second.max_iterations = options.max_iterations > phase1.iterations ? options.max_iterations - phase1.iterations : 1;
  EigshResult r = thick_restart(c64, second, &seed, k);
  r.fp32_iterations = phase1.iterations;
  r.fp64_iterations = r.iterations;
  r.iterations += phase1.iterations;
  r.reorthogonalization_passes += phase1.reorthogonalization_passes;
  r.conditional_second_passes += phase1.conditional_second_passes;
  r.operator_applications = c32.applications + c64.applications;
  return r;
}

}  // namespace qmbed
