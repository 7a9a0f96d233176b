// Batched Lanczos over sectors x scan points.
//
// Every (sector s, point p) pair is an independent Hermitian problem
// H(s, p) = sum_k c_k(p) A_k(s) whose lowest eigenvalues are wanted (the
// reference would call eigsh once per pair, src/solve/mod.rs:2335-2350). Here
// all pairs advance together: one column per pair in row-major blocks
// (rows of sector s) x (points), so one launch applies every sector's
// operator to every point, and the gather of a column reads all points of
// that row as one contiguous 512-byte or 1-KB line. The rows of all sectors are
// concatenated and each warp finds its sector by binary search, so sectors of
// uneven dimension share the launch.
//
// Method: the plain three-term Lanczos recurrence without reorthogonalisation
// (each column its own alpha, beta in FP64, all vectors FP64), in the
// orbit-scaled coordinates z = x / sqrt(R) with R-weighted inner products.
// Loss of orthogonality only adds copies of converged Ritz values; the
// lowest distinct Ritz values are taken after merging copies closer than
// 1e-8 max(|theta|, 1), and a pair is converged when its wanted values move
// by less than 1e-3 tol max(|theta|, 1) over `kCheck` steps. The tridiagonal
// eigenvalues come from Sturm-sequence bisection on the GPU, one thread per
// pair, from the alpha/beta histories kept in device memory.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "batched.cuh"

namespace qmbed {

namespace {

constexpr int kMaxComp = 8;
constexpr int kMaxSectors = 128;
constexpr int kRowsPerBlock = 256;  // reduction blocks: 8 warps x 32 rows
constexpr int kCheck = 10;
constexpr int kLowest = 8;  // Ritz values computed per pair at a check

struct CompRows {
  const void* row_ptr;
  const uint32_t* cols;
  const double* vals;
  const double* diag;
  int row_ptr64;
  int diag_complex;
};

struct SectorDesc {
  uint64_t row0, n, block0, blocks;
  const uint16_t* weights;
  double* buf[3];
  CompRows comp[kMaxComp];
};

__device__ __forceinline__ int find_sector(const uint64_t* starts, int ns, uint64_t g) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (starts[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint64_t row_begin(const CompRows& c, uint64_t r) {
  return c.row_ptr64 ? static_cast<const uint64_t*>(c.row_ptr)[r] : static_cast<const uint32_t*>(c.row_ptr)[r];
}

// out = H(s, p) cur - beta_prev(s, p) prev, one warp per row, lane owns PPL points
template <int PPL>
__global__ void __launch_bounds__(256) scan_apply_kernel(const SectorDesc* __restrict__ sec, int ns,
                                                         uint64_t total_rows, int K, const double* __restrict__ coef,
                                                         int cur, int prev, int out,
                                                         const double* __restrict__ beta_prev) {
  constexpr int P = 32 * PPL;
  __shared__ double c[kMaxComp * P];
  __shared__ uint64_t starts[kMaxSectors];
  for (int i = threadIdx.x; i < K * P; i += blockDim.x) c[i] = coef[i];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) starts[i] = sec[i].row0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < total_rows; g += warps) {
    const int s = find_sector(starts, ns, g);
    const SectorDesc& d = sec[s];
    const uint64_t r = g - d.row0;
    const double* z = d.buf[cur];
    double are[PPL], aim[PPL], dsum[PPL];
#pragma unroll
    for (int q = 0; q < PPL; ++q) are[q] = aim[q] = dsum[q] = 0.0;
    for (int k = 0; k < K; ++k) {
      const CompRows& cr = d.comp[k];
      double ck[PPL];
#pragma unroll
      for (int q = 0; q < PPL; ++q) ck[q] = c[k * P + lane * PPL + q];
      const uint64_t begin = row_begin(cr, r), end = row_begin(cr, r + 1);
      for (uint64_t e = begin; e < end; ++e) {
        const uint64_t col = cr.cols[e];
        const double vr = cr.vals[2 * e], vi = cr.vals[2 * e + 1];
        const double2* zc = reinterpret_cast<const double2*>(z) + col * P + lane * PPL;
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
          const double2 x = zc[q];
          are[q] = fma(ck[q], vr * x.x - vi * x.y, are[q]);
          aim[q] = fma(ck[q], vr * x.y + vi * x.x, aim[q]);
        }
      }
      const double dr = cr.diag_complex ? cr.diag[2 * r] : cr.diag[r];
#pragma unroll
      for (int q = 0; q < PPL; ++q) dsum[q] = fma(ck[q], dr, dsum[q]);
    }
    const double2* zs = reinterpret_cast<const double2*>(z) + r * P + lane * PPL;
    const double2* pv = reinterpret_cast<const double2*>(d.buf[prev]) + r * P + lane * PPL;
    double2* o = reinterpret_cast<double2*>(d.buf[out]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const double2 x = zs[q];
      double wr = are[q] + dsum[q] * x.x, wi = aim[q] + dsum[q] * x.y;
      if (beta_prev) {
        const double b = beta_prev[static_cast<uint64_t>(s) * P + lane * PPL + q];
        const double2 y = pv[q];
        wr -= b * y.x;
        wi -= b * y.y;
      }
      o[q] = make_double2(wr, wi);
    }
  }
}

// Reduction blocks: rows [b * kRowsPerBlock, ...) of one sector.
// MODE 0: partial[b][p] = sum_r R_r Re(conj(a) b)        (alpha)
// MODE 1: a -= alpha(s, p) b; partial = sum_r R_r |a|^2  (update + beta^2; alpha may be null)
template <int PPL, int MODE>
__global__ void __launch_bounds__(256) scan_reduce_kernel(const SectorDesc* __restrict__ sec, int ns, int ia, int ib,
                                                          const double* __restrict__ alpha,
                                                          double* __restrict__ partial) {
  constexpr int P = 32 * PPL;
  __shared__ uint64_t bstarts[kMaxSectors];
  __shared__ double red[8][P];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) bstarts[i] = sec[i].block0;
  __syncthreads();
  const int s = find_sector(bstarts, ns, blockIdx.x);
  const SectorDesc& d = sec[s];
  const uint64_t local_block = blockIdx.x - d.block0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[PPL];
#pragma unroll
  for (int q = 0; q < PPL; ++q) acc[q] = 0.0;
  double al[PPL];
#pragma unroll
  for (int q = 0; q < PPL; ++q) al[q] = (MODE == 1 && alpha) ? alpha[static_cast<uint64_t>(s) * P + lane * PPL + q] : 0.0;
  const uint64_t r0 = local_block * kRowsPerBlock;
  for (int i = warp; i < kRowsPerBlock; i += 8) {
    const uint64_t r = r0 + i;
    if (r >= d.n) break;
    const double w = d.weights ? static_cast<double>(d.weights[r]) : 1.0;
    double2* a = reinterpret_cast<double2*>(d.buf[ia]) + r * P + lane * PPL;
    const double2* b = reinterpret_cast<const double2*>(d.buf[ib]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      double2 x = a[q];
      const double2 y = b[q];
      if (MODE == 0) {
        acc[q] = fma(w, x.x * y.x + x.y * y.y, acc[q]);
      } else {
        x.x -= al[q] * y.x;
        x.y -= al[q] * y.y;
        if (alpha) a[q] = x;
        acc[q] = fma(w, x.x * x.x + x.y * x.y, acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < PPL; ++q) red[warp][lane * PPL + q] = acc[q];
  __syncthreads();
  if (threadIdx.x < P) {
    double t = 0.0;
    for (int w8 = 0; w8 < 8; ++w8) t += red[w8][threadIdx.x];
    partial[static_cast<uint64_t>(blockIdx.x) * P + threadIdx.x] = t;
  }
}

// out[s][p] = sum over sector s's blocks of partial (in block order); SQRT: sqrt
// of it, and the first step whose beta falls below 1e-12 (scale) is recorded.
__global__ void scan_finish_kernel(const SectorDesc* __restrict__ sec, int ns, int P, const double* __restrict__ partial,
                                   double* __restrict__ out, int sqrt_mode, int* __restrict__ length, int step,
                                   const double* __restrict__ alpha) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * P) return;
  const int s = t / P, p = t % P;
  double v = 0.0;
  for (uint64_t b = sec[s].block0; b < sec[s].block0 + sec[s].blocks; ++b) v += partial[b * P + p];
  if (sqrt_mode) {
    v = sqrt(fmax(v, 0.0));
    const double scale = alpha ? fmax(fabs(alpha[t]), 1.0) : 1.0;
    if (length && length[t] < 0 && v <= 1.0e-12 * scale) length[t] = step + 1;
  }
  out[t] = v;
}

// dst = src / beta(s, p) (0 where beta is 0)
template <int PPL>
__global__ void scan_scale_kernel(const SectorDesc* __restrict__ sec, int ns, uint64_t total_rows, int isrc, int idst,
                                  const double* __restrict__ beta) {
  constexpr int P = 32 * PPL;
  __shared__ uint64_t starts[kMaxSectors];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) starts[i] = sec[i].row0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < total_rows; g += warps) {
    const int s = find_sector(starts, ns, g);
    const SectorDesc& d = sec[s];
    const uint64_t r = g - d.row0;
    const double2* a = reinterpret_cast<const double2*>(d.buf[isrc]) + r * P + lane * PPL;
    double2* o = reinterpret_cast<double2*>(d.buf[idst]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const double b = beta[static_cast<uint64_t>(s) * P + lane * PPL + q];
      const double inv = b > 1.0e-300 ? 1.0 / b : 0.0;
      const double2 x = a[q];
      o[q] = make_double2(x.x * inv, x.y * inv);
    }
  }
}

// start vectors: real parts uniform in [-0.5, 0.5) from a splitmix64 hash of (seed, sector, point, row)
template <int PPL>
__global__ void scan_init_kernel(const SectorDesc* __restrict__ sec, int ns, uint64_t total_rows, int idst,
                                 uint64_t seed) {
  constexpr int P = 32 * PPL;
  __shared__ uint64_t starts[kMaxSectors];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) starts[i] = sec[i].row0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < total_rows; g += warps) {
    const int s = find_sector(starts, ns, g);
    const SectorDesc& d = sec[s];
    const uint64_t r = g - d.row0;
    double2* o = reinterpret_cast<double2*>(d.buf[idst]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      uint64_t z = seed ^ (0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(s) * 4096 + lane * PPL + q + 1)) ^ (r * 0xd1b54a32d192ed03ULL);
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      z ^= z >> 31;
      o[q] = make_double2(static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0) - 0.5, 0.0);
    }
  }
}

// Lowest `m_out` eigenvalues of each pair's tridiagonal T (alpha_j, beta_j for
// j < length) by Sturm bisection; one thread per pair.
__global__ void scan_tridiagonal_kernel(int cols, int steps, const double* __restrict__ alpha_hist,
                                        const double* __restrict__ beta_hist, const int* __restrict__ length,
                                        int m_out, double* __restrict__ values) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cols) return;
  int m = steps;
  if (length[t] > 0 && length[t] < m) m = length[t];
  auto a = [&](int j) { return alpha_hist[static_cast<size_t>(j) * cols + t]; };
  auto b = [&](int j) { return beta_hist[static_cast<size_t>(j) * cols + t]; };
  double lo = 1e300, hi = -1e300;
  for (int j = 0; j < m; ++j) {
    const double off = (j > 0 ? fabs(b(j - 1)) : 0.0) + (j + 1 < m ? fabs(b(j)) : 0.0);
    lo = fmin(lo, a(j) - off);
    hi = fmax(hi, a(j) + off);
  }
  auto count_below = [&](double x) {
    int c = 0;
    double q = a(0) - x;
    if (q < 0) ++c;
    for (int j = 1; j < m; ++j) {
      if (q == 0.0) q = 1e-300;
      const double bb = b(j - 1);
      q = a(j) - x - bb * bb / q;
      if (q < 0) ++c;
    }
    return c;
  };
  for (int i = 0; i < m_out; ++i) {
    if (i >= m) {
      values[static_cast<size_t>(t) * m_out + i] = NAN;
      continue;
    }
    double l = lo, h = hi;
    for (int it = 0; it < 200 && h - l > 4.0e-16 * fmax(fabs(l), fabs(h)) + 1e-300; ++it) {
      const double mid = 0.5 * (l + h);
      if (count_below(mid) > i) h = mid;
      else l = mid;
    }
    values[static_cast<size_t>(t) * m_out + i] = 0.5 * (l + h);
  }
}

template <typename F>
void by_points(int P, F&& f) {
  if (P == 32) f(std::integral_constant<int, 1>{});
  else f(std::integral_constant<int, 2>{});
}

}  // namespace

ScanResult scan_lowest(const std::vector<std::vector<const SpinOperator*>>& components,
                       const std::vector<double>& coefficients, int points, int eigenpairs, double tolerance,
                       int max_steps, uint64_t seed, BlockOps& ops) {
  const int ns = static_cast<int>(components.size());
  if (ns < 1 || ns > kMaxSectors) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 128 sectors");
  const int K = static_cast<int>(components[0].size());
  if (K < 1 || K > kMaxComp) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 8 components");
  if (points < 1 || points > 64) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 64 points");
  if (eigenpairs < 1 || eigenpairs > 4) raise(QMBED_INVALID_OPTIONS, "a scan returns 1 to 4 eigenvalues per pair");
  if (!(tolerance > 0.0) || max_steps < 1) raise(QMBED_INVALID_OPTIONS, "tolerance and steps must be positive");
  if (static_cast<int>(coefficients.size()) != points * K) raise(QMBED_DIMENSION_MISMATCH, "coefficients must be points x components");
  const int P = points <= 32 ? 32 : 64;
  const cudaStream_t stream = ops.stream();
  // coefficients padded to P columns by repeating the last point
  std::vector<double> coef(static_cast<size_t>(K) * P);
  for (int k = 0; k < K; ++k)
    for (int p = 0; p < P; ++p) coef[static_cast<size_t>(k) * P + p] = coefficients[static_cast<size_t>(std::min(p, points - 1)) * K + k];
  std::vector<SectorDesc> desc(ns);
  uint64_t rows = 0, blocks = 0;
  size_t block_bytes_total = 0;
  for (int s = 0; s < ns; ++s) {
    if (static_cast<int>(components[s].size()) != K) raise(QMBED_DIMENSION_MISMATCH, "every sector needs the same components");
    const SpinOperator* first = components[s][0];
    SectorDesc& d = desc[s];
    std::memset(&d, 0, sizeof(d));
    d.n = first->dim();
    d.row0 = rows;
    d.block0 = blocks;
    d.blocks = (d.n + kRowsPerBlock - 1) / kRowsPerBlock;
    d.weights = first->basis().symmetric() ? first->basis().orbits() : nullptr;
    rows += d.n;
    blocks += d.blocks;
    block_bytes_total += 3 * d.n * P * 16;
    for (int k = 0; k < K; ++k) {
      const SpinOperator* op = components[s][k];
      if (op->dim() != d.n || &op->basis() != &first->basis())
        raise(QMBED_DIMENSION_MISMATCH, "the components of a sector must share its basis");
      const SpinOperator::ExplicitRows er = op->explicit_rows();
      d.comp[k] = CompRows{er.row_ptr, er.cols, er.values, er.diag, er.row_ptr64 ? 1 : 0, er.diag_complex ? 1 : 0};
    }
  }
  const int cols = ns * P;
  DeviceBuffer blocks_mem(block_bytes_total), desc_dev(ns * sizeof(SectorDesc)), coef_dev(coef.size() * sizeof(double));
  DeviceBuffer partial(std::max<uint64_t>(blocks, 1) * P * sizeof(double));
  DeviceBuffer alpha_hist(static_cast<size_t>(max_steps) * cols * sizeof(double));
  DeviceBuffer beta_hist(static_cast<size_t>(max_steps + 1) * cols * sizeof(double));
  DeviceBuffer length(cols * sizeof(int)), ritz(static_cast<size_t>(cols) * kLowest * sizeof(double));
  size_t offset = 0;
  for (int s = 0; s < ns; ++s)
    for (int b = 0; b < 3; ++b) {
      desc[s].buf[b] = reinterpret_cast<double*>(static_cast<char*>(blocks_mem.get()) + offset);
      offset += desc[s].n * P * 16;
    }
  QMBED_CUDA(cudaMemcpyAsync(desc_dev.get(), desc.data(), ns * sizeof(SectorDesc), cudaMemcpyHostToDevice, stream));
  QMBED_CUDA(cudaMemcpyAsync(coef_dev.get(), coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  QMBED_CUDA(cudaMemsetAsync(length.get(), 0xff, cols * sizeof(int), stream));  // -1: no breakdown yet
  const SectorDesc* sd = desc_dev.as<SectorDesc>();
  const int row_grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((rows * 32 + 255) / 256, 16ull * ops.sms())));
  const int red_grid = static_cast<int>(blocks);
  const int fin_grid = (cols + 127) / 128;
  double* beta0 = beta_hist.as<double>() + static_cast<size_t>(max_steps) * cols;  // start-vector norms

  ScanResult result;
  result.eigenvalues.assign(static_cast<size_t>(ns) * points * eigenpairs, std::nan(""));
  result.steps.assign(static_cast<size_t>(ns) * points, -1);
  by_points(P, [&](auto ptag) {
    constexpr int PPL = decltype(ptag)::value;
    int cur = 0, prev = 1, work = 2;
    // normalised start vectors in buffer `cur`
    scan_init_kernel<PPL><<<row_grid, 256, 0, stream>>>(sd, ns, rows, work, seed);
    scan_reduce_kernel<PPL, 1><<<red_grid, 256, 0, stream>>>(sd, ns, work, work, nullptr, partial.as<double>());
    scan_finish_kernel<<<fin_grid, 128, 0, stream>>>(sd, ns, P, partial.as<double>(), beta0, 1, nullptr, 0, nullptr);
    scan_scale_kernel<PPL><<<row_grid, 256, 0, stream>>>(sd, ns, rows, work, cur, beta0);
    QMBED_LAUNCH_CHECK();
    std::vector<double> previous(static_cast<size_t>(cols) * eigenpairs, std::nan("")), host(static_cast<size_t>(cols) * kLowest);
    std::vector<int> host_len(cols);
    std::vector<char> done(cols, 0);
    int active = cols;
    for (int j = 0; j < max_steps && active > 0; ++j) {
      double* alpha_j = alpha_hist.as<double>() + static_cast<size_t>(j) * cols;
      double* beta_j = beta_hist.as<double>() + static_cast<size_t>(j) * cols;
      const double* beta_prev = j > 0 ? beta_hist.as<double>() + static_cast<size_t>(j - 1) * cols : nullptr;
      scan_apply_kernel<PPL><<<row_grid, 256, 0, stream>>>(sd, ns, rows, K, coef_dev.as<double>(), cur, prev, work, beta_prev);
      scan_reduce_kernel<PPL, 0><<<red_grid, 256, 0, stream>>>(sd, ns, cur, work, nullptr, partial.as<double>());
      scan_finish_kernel<<<fin_grid, 128, 0, stream>>>(sd, ns, P, partial.as<double>(), alpha_j, 0, nullptr, j, nullptr);
      scan_reduce_kernel<PPL, 1><<<red_grid, 256, 0, stream>>>(sd, ns, work, cur, alpha_j, partial.as<double>());
      scan_finish_kernel<<<fin_grid, 128, 0, stream>>>(sd, ns, P, partial.as<double>(), beta_j, 1, length.as<int>(), j, alpha_j);
      scan_scale_kernel<PPL><<<row_grid, 256, 0, stream>>>(sd, ns, rows, work, prev, beta_j);
      QMBED_LAUNCH_CHECK();
      std::swap(cur, prev);  // the new vector went to the old prev buffer
      result.total_steps = j + 1;
      if ((j + 1) % kCheck != 0 && j + 1 != max_steps) continue;
      scan_tridiagonal_kernel<<<fin_grid, 128, 0, stream>>>(cols, j + 1, alpha_hist.as<double>(), beta_hist.as<double>(),
                                                            length.as<int>(), kLowest, ritz.as<double>());
      QMBED_LAUNCH_CHECK();
      QMBED_CUDA(cudaMemcpyAsync(host.data(), ritz.get(), host.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
      QMBED_CUDA(cudaMemcpyAsync(host_len.data(), length.get(), cols * sizeof(int), cudaMemcpyDeviceToHost, stream));
      QMBED_CUDA(cudaStreamSynchronize(stream));
      for (int c = 0; c < cols; ++c) {
        if (done[c]) continue;
        // lowest distinct Ritz values (copies from lost orthogonality merged)
        std::vector<double> distinct;
        for (int i = 0; i < kLowest && static_cast<int>(distinct.size()) < eigenpairs; ++i) {
          const double v = host[static_cast<size_t>(c) * kLowest + i];
          if (std::isnan(v)) break;
          if (distinct.empty() || v - distinct.back() > 1.0e-8 * std::max(std::fabs(v), 1.0)) distinct.push_back(v);
        }
        const bool exhausted = host_len[c] > 0;
        bool converged = static_cast<int>(distinct.size()) == eigenpairs || exhausted;
        for (int i = 0; i < eigenpairs && converged; ++i) {
          if (i >= static_cast<int>(distinct.size())) break;
          const double old = previous[static_cast<size_t>(c) * eigenpairs + i];
          if (!exhausted && !(std::fabs(distinct[i] - old) <= 1.0e-3 * tolerance * std::max(std::fabs(distinct[i]), 1.0)))
            converged = false;
        }
        for (int i = 0; i < eigenpairs; ++i)
          previous[static_cast<size_t>(c) * eigenpairs + i] = i < static_cast<int>(distinct.size()) ? distinct[i] : std::nan("");
        if (!converged) continue;
        done[c] = 1;
        --active;
        const int s = c / P, p = c % P;
        if (p >= points) continue;
        result.steps[static_cast<size_t>(s) * points + p] = exhausted ? std::min(j + 1, host_len[c]) : j + 1;
        result.applications += static_cast<size_t>(j + 1);
        for (int i = 0; i < eigenpairs && i < static_cast<int>(distinct.size()); ++i)
          result.eigenvalues[(static_cast<size_t>(s) * points + p) * eigenpairs + i] = distinct[i];
      }
    }
  });
  for (size_t i = 0; i < result.steps.size(); ++i)
    if (result.steps[i] < 0) raise_nonconvergence(static_cast<size_t>(result.total_steps), std::nan(""));
  return result;
}

}  // namespace qmbed
