// Block Chebyshev-filtered subspace iteration for the smallest algebraic
// eigenpairs of a real Hermitian operator.
//
// Method: the scaled Chebyshev filter recurrence of Zhou, Saad, Tiago and
// Chelikowsky (J. Comput. Phys. 219, 2006, Algorithm 4.1 "scaled"), followed
// by an orthonormalisation of the block through the eigen-decomposition of its
// Gram matrix and a Rayleigh-Ritz step. The filter interval [cut, upper] is
// damped, everything below `cut` is amplified. `upper` comes from a short
// Lanczos run: the largest Ritz value plus the residual norm of its Ritz pair
// and 1% of the Ritz range (after the bound estimators of Zhou and Li, Linear
// Algebra Appl. 435, 2011); `cut` is the largest Ritz value of the block (by
// interlacing it lies at or above the block's share of the spectrum). The
// filter degree per outer iteration follows the estimated convergence rate
// acosh((c - theta_i) / e) of the slowest wanted pair, capped so that the
// Gram-based orthonormalisation keeps the weakest block direction.
//
// All block work happens in the orbit-scaled coordinates z = S^-1 x,
// S = diag(sqrt(R)): the packed rows then need no orbit factor, inner products
// carry the weight R (x.y = sum_r R_r z_r w_r) and the eigenvectors are x = S z.
// Blocks are row-major n x nb so that one gathered column is one contiguous
// 32/64-byte read for all nb vectors.
//
// Precision: FP32 blocks and block action (FP32 accumulation) with FP64 Gram
// and Ritz matrices until every wanted residual is below 1e-5 of max(|lambda|,1)
// (or stops improving), then FP64 blocks to the requested tolerance. The
// acceptance test is the reference's r <= tol * max(|lambda|, 1)
// (src/solve/mod.rs:1255, 1863), with r = ||H x - lambda x|| for ||x|| = 1.
// The small symmetric eigenproblems run on the GPU (device Jacobi).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <numeric>
#include <type_traits>
#include <vector>

#include "device_util.cuh"
#include <string>

#include "filtered.cuh"

namespace qmbed {

namespace {

constexpr int kThreads = 256;
constexpr int kGramElems = 2048;            // block elements staged per tile of the Gram kernel
constexpr double kFilterHandover = 1.0e-5;  // FP32 phase target (relative residual)
constexpr int kMaxOuter = 80;               // outer iterations per precision phase
constexpr int kBoundSteps = 24;             // Lanczos steps of the spectral bound estimate
constexpr int kMaxDegree = 60;
constexpr size_t kMaxFilteredPairs = 12;
constexpr uint64_t kMinFilteredDim = 1024;

// partial[b][i * NB + j] = sum over the rows of block b of w_r a[r][i] b[r][j]  (FP64)
template <typename T, int NB>
__global__ void __launch_bounds__(kThreads) block_gram_kernel(uint64_t n, const T* __restrict__ a,
                                                               const T* __restrict__ b,
                                                               const uint16_t* __restrict__ weights,
                                                               double* __restrict__ partial) {
  constexpr int kRows = kGramElems / NB;
  constexpr int kPairs = NB * NB;
  constexpr int kSplit = kThreads / kPairs;
  static_assert(kThreads % kPairs == 0, "pairs must divide the block");
  __shared__ double sa[kGramElems];
  __shared__ double sb[kGramElems];
  __shared__ double red[kThreads];
  const int pair = threadIdx.x % kPairs, sub = threadIdx.x / kPairs;
  const int i = pair / NB, j = pair % NB;
  const uint64_t limit = n * NB;
  double acc = 0.0;
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kRows; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * kRows) {
    const uint64_t base = t0 * NB;
#pragma unroll
    for (int q = 0; q < kGramElems / kThreads; ++q) {
      const int e = q * kThreads + threadIdx.x;
      const uint64_t g = base + e;
      double va = 0.0, vb = 0.0;
      if (g < limit) {
        const double w = weights ? static_cast<double>(weights[t0 + e / NB]) : 1.0;
        va = w * static_cast<double>(a[g]);
        vb = static_cast<double>(b[g]);
      }
      sa[e] = va;
      sb[e] = vb;
    }
    __syncthreads();
    for (int r = sub; r < kRows; r += kSplit) acc += sa[r * NB + i] * sb[r * NB + j];
    __syncthreads();
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < kPairs) {
    double s = 0.0;
    for (int q = 0; q < kSplit; ++q) s += red[q * kPairs + threadIdx.x];
    partial[static_cast<uint64_t>(blockIdx.x) * kPairs + threadIdx.x] = s;
  }
}

// D = A B + C on the FP64 tensor cores: one m8n8k4 MMA per warp, A 8 x 4
// (row major), B 4 x 8 (column major). Per lane: a = A[lane / 4][lane % 4],
// b = B[lane % 4][lane / 4], c/d = C[lane / 4][2 (lane % 4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double a, double b, double& c0, double& c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// The same weighted Gram on the tensor cores. The contraction runs over the
// rows: every MMA takes 4 consecutive rows of the row-major n x NB blocks, so
// the 32 lanes' operand loads are the 4 x 8 sub-block of a and of b (one
// contiguous 256-byte (FP64) or 128-byte (FP32) span per operand). A warp
// keeps the (NB / 8)^2 output tiles of the NB x NB Gram in registers, strides
// over groups of 4 rows, and the block reduces its warps in a fixed order.
template <typename T, int NB>
__global__ void __launch_bounds__(kThreads) block_gram_mma_kernel(uint64_t n, const T* __restrict__ a,
                                                                   const T* __restrict__ b,
                                                                   const uint16_t* __restrict__ weights,
                                                                   double* __restrict__ partial) {
  constexpr int TILES = NB / 8;
  constexpr int kWarps = kThreads / 32;
  constexpr int kUnroll = 4;  // row groups whose operands are loaded before their MMAs
  __shared__ double red[kWarps][NB * NB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kr = lane & 3, col = lane >> 2;  // operand row within the group, column within a tile
  double c[TILES][TILES][2];
#pragma unroll
  for (int p = 0; p < TILES; ++p)
#pragma unroll
    for (int q = 0; q < TILES; ++q) c[p][q][0] = c[p][q][1] = 0.0;
  const uint64_t groups = (n + 3) / 4;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kWarps;
  for (uint64_t g0 = static_cast<uint64_t>(blockIdx.x) * kWarps + warp; g0 < groups; g0 += stride * kUnroll) {
    double va[kUnroll][TILES], vb[kUnroll][TILES];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint64_t g = g0 + u * stride;
      const uint64_t r = g * 4 + kr;
      const bool in = g < groups && r < n;
      const double w = in ? (weights ? static_cast<double>(__ldg(weights + r)) : 1.0) : 0.0;
#pragma unroll
      for (int t = 0; t < TILES; ++t) {
        va[u][t] = in ? w * static_cast<double>(__ldg(a + r * NB + t * 8 + col)) : 0.0;
        vb[u][t] = in ? static_cast<double>(__ldg(b + r * NB + t * 8 + col)) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int p = 0; p < TILES; ++p)
#pragma unroll
        for (int q = 0; q < TILES; ++q) dmma_8x8x4(va[u][p], vb[u][q], c[p][q][0], c[p][q][1]);
  }
#pragma unroll
  for (int p = 0; p < TILES; ++p)
#pragma unroll
    for (int q = 0; q < TILES; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) red[warp][(p * 8 + col) * NB + q * 8 + 2 * kr + h] = c[p][q][h];
  __syncthreads();
  for (int t = threadIdx.x; t < NB * NB; t += kThreads) {
    double s = 0.0;
    for (int w8 = 0; w8 < kWarps; ++w8) s += red[w8][t];
    partial[static_cast<uint64_t>(blockIdx.x) * NB * NB + t] = s;
  }
}

// out[t] = sum_b partial[b][t] in block order (deterministic).
__global__ void reduce_partials_kernel(const double* __restrict__ partial, int blocks, int count,
                                       double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b) s += partial[static_cast<size_t>(b) * count + t];
  out[t] = s;
}

// out[r][:] = z[r][:] C (C row-major NB x NB, FP64 arithmetic; out must not
// alias z). With RESID also
// partial[b][q] = sum_r w_r ((w[r][:] C)_q - theta_q out[r][q])^2.
// Each thread produces 8 outputs of one row (NB / 8 threads per row), which
// keeps the per-thread state near 100 registers instead of hoisting all of C.
template <typename T, int NB, bool RESID>
__global__ void __launch_bounds__(kThreads, 2) block_rotate_kernel(uint64_t n, const T* __restrict__ z,
                                                                    T* __restrict__ out, const T* __restrict__ w,
                                                                    const double* __restrict__ coeff,
                                                                    const double* __restrict__ theta,
                                                                    const uint16_t* __restrict__ weights,
                                                                    double* __restrict__ partial) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr int OUT = 8;
  constexpr int SPLIT = NB / OUT;
  static_assert(NB % OUT == 0 && 32 % SPLIT == 0, "rows must split evenly across lanes");
  __shared__ double c[NB * NB];
  __shared__ double th[NB];
  __shared__ double red[kThreads / 32][NB];
  for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) c[i] = coeff[i];
  if (RESID)
    for (int i = threadIdx.x; i < NB; i += blockDim.x) th[i] = theta[i];
  __syncthreads();
  double res[OUT];
#pragma unroll
  for (int q = 0; q < OUT; ++q) res[q] = 0.0;
  // the grid stride is a multiple of SPLIT, so a thread keeps its part
  const int part = static_cast<int>(threadIdx.x % SPLIT);
  const uint64_t total = n * SPLIT;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t r = t / SPLIT;
    double zin[NB];
#pragma unroll
    for (int v = 0; v < NB; v += VEC) {
      T x[VEC];
      load16(z + r * NB + v, x);
#pragma unroll
      for (int q = 0; q < VEC; ++q) zin[v + q] = static_cast<double>(x[q]);
    }
    double zo[OUT];
#pragma unroll
    for (int q = 0; q < OUT; ++q) {
      const int col = part * OUT + q;
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < NB; ++j) s = fma(zin[j], c[j * NB + col], s);
      zo[q] = s;
    }
#pragma unroll
    for (int v = 0; v < OUT; v += VEC) {
      T x[VEC];
#pragma unroll
      for (int q = 0; q < VEC; ++q) x[q] = static_cast<T>(zo[v + q]);
      store16(out + r * NB + part * OUT + v, x);
    }
    if (RESID) {
      double win[NB];
#pragma unroll
      for (int v = 0; v < NB; v += VEC) {
        T x[VEC];
        load16(w + r * NB + v, x);
#pragma unroll
        for (int q = 0; q < VEC; ++q) win[v + q] = static_cast<double>(x[q]);
      }
      const double wr = weights ? static_cast<double>(weights[r]) : 1.0;
#pragma unroll
      for (int q = 0; q < OUT; ++q) {
        const int col = part * OUT + q;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j) s = fma(win[j], c[j * NB + col], s);
        const double d = s - th[col] * zo[q];
        res[q] = fma(wr * d, d, res[q]);
      }
    }
  }
  if (RESID) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < OUT; ++q) {
      double v = res[q];
      for (int o = 16; o >= SPLIT; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane < SPLIT) red[warp][lane * OUT + q] = v;
    }
    __syncthreads();
    if (threadIdx.x < NB) {
      double s = 0.0;
      for (int q = 0; q < kThreads / 32; ++q) s += red[q][threadIdx.x];
      partial[static_cast<uint64_t>(blockIdx.x) * NB + threadIdx.x] = s;
    }
  }
}

// out[i * n + r] = sqrt(R_r) z[r][i] for i < k (FP64, column-major).
template <typename T, int NB>
__global__ void block_export_kernel(uint64_t n, const T* __restrict__ z, int k, const uint16_t* __restrict__ weights,
                                    double* __restrict__ out) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const double s = weights ? sqrt(static_cast<double>(weights[r])) : 1.0;
    for (int i = 0; i < k; ++i) out[static_cast<uint64_t>(i) * n + r] = s * static_cast<double>(z[r * NB + i]);
  }
}

// z[r][i] = cols[i * n + r] / sqrt(R_r) for i < NB (FP64 column-major input).
template <typename T, int NB>
__global__ void block_import_kernel(uint64_t n, const double* __restrict__ cols, const uint16_t* __restrict__ weights,
                                    T* __restrict__ z) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const double s = weights ? 1.0 / sqrt(static_cast<double>(weights[r])) : 1.0;
    for (int i = 0; i < NB; ++i) z[r * NB + i] = static_cast<T>(s * cols[static_cast<uint64_t>(i) * n + r]);
  }
}

template <typename F>
void dispatch_block(int prec, int nb, F&& f) {
  using NB8 = std::integral_constant<int, 8>;
  using NB16 = std::integral_constant<int, 16>;
  if (prec == 64) {
    if (nb == 8) f(double{}, NB8{});
    else f(double{}, NB16{});
  } else {
    if (nb == 8) f(float{}, NB8{});
    else f(float{}, NB16{});
  }
}

class BlockSolver {
 public:
  BlockSolver(const LinearOperatorView& op, const EigshOptions& o, BlockOps& ops, int nb)
      : op_(op), o_(o), ops_(ops), n_(op.dim), nb_(nb), blocks_(2 * ops.sms()) {
    partial_.allocate(static_cast<size_t>(blocks_) * 2 * nb * nb * sizeof(double));
    result_.allocate(static_cast<size_t>(nb) * nb * sizeof(double));
    coeff_.allocate((static_cast<size_t>(nb) * nb + nb) * sizeof(double));
  }

  size_t applications = 0;
  size_t block_actions = 0;

  // out = alpha * Ht z + beta * z + gamma * p
  void act(int prec, const void* z, const void* p, void* out, double alpha, double beta, double gamma) {
    op_.block_apply(prec, nb_, z, p, out, alpha, beta, gamma);
    applications += static_cast<size_t>(nb_);
    ++block_actions;
  }

  // G[i][j] = sum_r R_r a[r][i] b[r][j], on the FP64 tensor cores unless
  // QMBED_DENSE=scalar selects the CUDA-core kernel.
  std::vector<double> gram(int prec, const void* a, const void* b) {
    const cudaStream_t s = ops_.stream();
    const bool scalar = !dense_on_tensor_cores();
    dispatch_block(prec, nb_, [&](auto ttag, auto nbtag) {
      using T = decltype(ttag);
      constexpr int NB = decltype(nbtag)::value;
      if (scalar)
        block_gram_kernel<T, NB><<<blocks_, kThreads, 0, s>>>(n_, static_cast<const T*>(a), static_cast<const T*>(b),
                                                              op_.weights, partial_.as<double>());
      else
        block_gram_mma_kernel<T, NB><<<blocks_, kThreads, 0, s>>>(
            n_, static_cast<const T*>(a), static_cast<const T*>(b), op_.weights, partial_.as<double>());
    });
    QMBED_LAUNCH_CHECK();
    return reduce(nb_ * nb_);
  }

  // out = z C (out must not alias z); with `resid` returns the squared
  // weighted residual norms of (w C) - out diag(theta).
  std::vector<double> rotate(int prec, const void* z, void* out, const void* w, const std::vector<double>& C,
                             const std::vector<double>& theta, bool resid) {
    const cudaStream_t s = ops_.stream();
    std::vector<double> host(C);
    host.resize(static_cast<size_t>(nb_) * nb_ + nb_, 0.0);
    for (size_t q = 0; q < theta.size() && q < static_cast<size_t>(nb_); ++q) host[static_cast<size_t>(nb_) * nb_ + q] = theta[q];
    QMBED_CUDA(cudaMemcpyAsync(coeff_.get(), host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    const double* c = coeff_.as<double>();
    dispatch_block(prec, nb_, [&](auto ttag, auto nbtag) {
      using T = decltype(ttag);
      constexpr int NB = decltype(nbtag)::value;
      if (resid)
        block_rotate_kernel<T, NB, true><<<blocks_, kThreads, 0, s>>>(
            n_, static_cast<const T*>(z), static_cast<T*>(out), static_cast<const T*>(w), c, c + NB * NB,
            op_.weights, partial_.as<double>());
      else
        block_rotate_kernel<T, NB, false><<<blocks_, kThreads, 0, s>>>(
            n_, static_cast<const T*>(z), static_cast<T*>(out), nullptr, c, nullptr, op_.weights, nullptr);
    });
    QMBED_LAUNCH_CHECK();
    if (!resid) return {};
    return reduce(nb_);
  }

  // Orthonormal block (weighted inner product) spanning the columns of *A,
  // left in *A (B is scratch; the pointers may be exchanged).
  void orthonormalize(int prec, void*& A, void*& B, int passes) {
    for (int pass = 0; pass < passes; ++pass) {
      std::vector<double> G = gram(prec, A, A), mu, V;
      device_symmetric_eigen(nb_, G, mu, V, ops_.stream());
      const double top = std::max(mu.back(), std::numeric_limits<double>::min());
      const double floor = top * (prec == 64 ? 1.0e-28 : 1.0e-14);
      std::vector<double> C(static_cast<size_t>(nb_) * nb_);
      for (int j = 0; j < nb_; ++j)
        for (int q = 0; q < nb_; ++q) C[static_cast<size_t>(j) * nb_ + q] = V[static_cast<size_t>(j) * nb_ + q] / std::sqrt(std::max(mu[q], floor));
      rotate(prec, A, B, nullptr, C, {}, false);
      std::swap(A, B);
    }
  }

  // Rayleigh-Ritz on the orthonormal block *A (B, W scratch): *A becomes the
  // Ritz vectors, ascending values in theta, residual norms in res.
  void rayleigh_ritz(int prec, void*& A, void*& B, void* W, std::vector<double>& theta, std::vector<double>& res) {
    act(prec, A, nullptr, W, 1.0, 0.0, 0.0);
    std::vector<double> Tm = gram(prec, A, W), Y;
    device_symmetric_eigen(nb_, Tm, theta, Y, ops_.stream());
    std::vector<double> r2 = rotate(prec, A, B, W, Y, theta, true);
    std::swap(A, B);
    res.assign(nb_, 0.0);
    for (int q = 0; q < nb_; ++q) res[q] = std::sqrt(std::max(r2[q], 0.0));
  }

  // Scaled Chebyshev filter of degree d on [cut, upper] with spectrum lower
  // estimate `lower`; the block in *A is filtered, B is scratch. On return *A
  // holds the filtered block (the two pointers may be exchanged).
  void filter(int prec, void*& A, void*& B, int degree, double lower, double cut, double upper) {
    if (degree <= 0) return;
    const double e = 0.5 * (upper - cut), c = 0.5 * (upper + cut);
    const double sigma1 = e / (lower - c);
    double sigma = sigma1;
    act(prec, A, nullptr, B, sigma1 / e, -sigma1 * c / e, 0.0);
    void* prev = A;
    void* cur = B;
    for (int i = 2; i <= degree; ++i) {
      const double next = 1.0 / (2.0 / sigma1 - sigma);
      act(prec, cur, prev, prev, 2.0 * next / e, -2.0 * next * c / e, -sigma * next);
      std::swap(prev, cur);
      sigma = next;
    }
    A = cur;
    B = prev;
  }

  void import_columns(int prec, const double* cols, void* z) {
    const int G = std::max(1, std::min<int>(static_cast<int>((n_ + kThreads - 1) / kThreads), 8 * ops_.sms()));
    dispatch_block(prec, nb_, [&](auto ttag, auto nbtag) {
      using T = decltype(ttag);
      constexpr int NB = decltype(nbtag)::value;
      block_import_kernel<T, NB><<<G, kThreads, 0, ops_.stream()>>>(n_, cols, op_.weights, static_cast<T*>(z));
    });
    QMBED_LAUNCH_CHECK();
  }

  void export_columns(int prec, const void* z, int k, double* out) {
    const int G = std::max(1, std::min<int>(static_cast<int>((n_ + kThreads - 1) / kThreads), 8 * ops_.sms()));
    dispatch_block(prec, nb_, [&](auto ttag, auto nbtag) {
      using T = decltype(ttag);
      constexpr int NB = decltype(nbtag)::value;
      block_export_kernel<T, NB><<<G, kThreads, 0, ops_.stream()>>>(n_, static_cast<const T*>(z), k, op_.weights, out);
    });
    QMBED_LAUNCH_CHECK();
  }

 private:
  std::vector<double> reduce(int count) {
    const cudaStream_t s = ops_.stream();
    reduce_partials_kernel<<<(count + 127) / 128, 128, 0, s>>>(partial_.as<double>(), blocks_, count, result_.as<double>());
    QMBED_LAUNCH_CHECK();
    std::vector<double> host(count);
    QMBED_CUDA(cudaMemcpyAsync(host.data(), result_.get(), count * sizeof(double), cudaMemcpyDeviceToHost, s));
    QMBED_CUDA(cudaStreamSynchronize(s));
    return host;
  }

  const LinearOperatorView& op_;
  const EigshOptions& o_;
  BlockOps& ops_;
  uint64_t n_;
  int nb_;
  int blocks_;
  DeviceBuffer partial_, result_, coeff_;
};

struct Bounds {
  std::vector<double> theta;  // ascending Ritz values
  double beta = 0.0;          // last Lanczos beta
  double top_residual = 0.0;  // ||H y - theta_max y|| of the top Ritz pair
  int steps = 0;
};

// Spectral bounds from a short Lanczos run in FP32 without reorthogonalisation
// (only the extreme Ritz values are used). `start` is an FP64 real vector.
Bounds lanczos_bounds(const LinearOperatorView& op, BlockOps& ops, const double* start, size_t& applications,
                      int steps = kBoundSteps) {
  const uint64_t n = op.dim;
  const int m = static_cast<int>(std::min<uint64_t>(static_cast<uint64_t>(std::max(steps, 2)), n - 1));
  // workspace slots 7-9 of the handle: the three FP32 Lanczos vectors
  void* prev = ops.workspace(7, n * 4);
  void* cur = ops.workspace(8, n * 4);
  void* w_vec = ops.workspace(9, n * 4);
  ops.convert(start, 64, cur, 32, n);
  const double n0 = ops.norm(cur, n, 32, false);
  if (!(n0 > 0.0)) raise(QMBED_INVALID_OPTIONS, "eigsh start vector has zero norm");
  ops.scale(cur, n, n0, 32, false);
  std::vector<double> alpha, beta;
  double b_prev = 0.0;
  for (int j = 0; j < m; ++j) {
    op.apply(32, false, cur, w_vec);
    ++applications;
    C64 h;
    ops.dots(cur, n, 1, w_vec, n, 32, false, &h);
    double norm = ops.subtract(cur, n, 1, &h, w_vec, n, 32, false, j == 0);
    if (j > 0) {
      const C64 hb(b_prev, 0.0);
      norm = ops.subtract(prev, n, 1, &hb, w_vec, n, 32, false, true);
    }
    alpha.push_back(h.real());
    beta.push_back(norm);
    if (!(norm > 1.0e-10 * std::max(1.0, std::fabs(h.real())))) break;
    std::swap(prev, cur);
    ops.scale_into(w_vec, cur, n, norm, 32, false);
    b_prev = norm;
  }
  const int size = static_cast<int>(alpha.size());
  std::vector<double> vals, vecs;
  tridiagonal_eigen(alpha, std::vector<double>(beta.begin(), beta.begin() + (size - 1)), false, vals, vecs);
  // residual norm of the top Ritz pair: |beta_m| times the last component of its vector
  const double top_residual = std::fabs(beta.back() * vecs[static_cast<size_t>(size - 1) * size + (size - 1)]);
  return Bounds{vals, beta.back(), top_residual, size};
}

}  // namespace

bool filtered_applicable(const LinearOperatorView& op, const EigshOptions& o, bool complex_initial) {
  return static_cast<bool>(op.block_apply) && op.real && !complex_initial && o.target == kSmallestAlgebraic &&
         o.eigenpairs <= kMaxFilteredPairs && op.dim >= kMinFilteredDim;
}

EigshResult filtered_eigsh(const LinearOperatorView& op, const EigshOptions& o, const double* staged_initial,
                           int n_initial, BlockOps& ops) {
  const uint64_t n = op.dim;
  const int k = static_cast<int>(o.eigenpairs);
  const int nb = k <= 5 ? 8 : 16;
  BlockSolver solver(op, o, ops, nb);

  // Start columns: the caller's vectors (real parts), then reference
  // deterministic starts with seeds o.seed + j * 0x9e3779b9 for the remaining
  // column positions j (a caller's vector equal to the default start of
  // column 0 is then not repeated).
  // Workspace slots of the handle: 0 start columns, 1-3 FP32 blocks, 4-6 FP64
  // blocks, 7-9 the bound estimate's Lanczos vectors.
  const size_t block32 = static_cast<size_t>(n) * nb * 4, block64 = static_cast<size_t>(n) * nb * 8;
  double* cols = static_cast<double*>(ops.workspace(0, block64));
  auto col = [&](int j) { return cols + static_cast<size_t>(j) * n; };
  const int used = std::min(n_initial, nb);
  for (int j = 0; j < used; ++j) ops.import_complex(staged_initial + 2 * static_cast<size_t>(j) * n, col(j), n, 64, false);
  for (int j = used; j < nb; ++j) ops.lcg_start(col(j), n, o.seed + static_cast<uint64_t>(j) * 0x9e3779b9ULL, 64, false);

  // QMBED_FILTER_TRACE=1 prints one line per outer iteration to stderr
  const char* trace_env = std::getenv("QMBED_FILTER_TRACE");
  const bool trace = trace_env && trace_env[0] == '1';
  const auto started = std::chrono::steady_clock::now();
  auto stamp = [&](const char* what) {
    if (!trace) return;
    ops.sync();
    std::fprintf(stderr, "[filter] %s at %.1f ms\n", what,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - started).count());
  };
  size_t bound_applications = 0;
  // The bound runs start from a deterministic start column: a caller's
  // vectors may be near eigenvectors (a refinement), from which a short
  // Lanczos run sees little of the spectrum.
  const double* bound_start = col(used < nb ? used : 0);
  // A spectral hint replaces the bound estimate when the Ritz values of a
  // short check run lie inside its interval (Ritz values lie inside the
  // spectrum, so an interval that misses one is wrong).
  bool hint_used = false;
  Bounds bd;
  if (o.hint && o.hint_upper > o.hint_lower) {
    bd = lanczos_bounds(op, ops, bound_start, bound_applications, o.hint_check_steps);
    hint_used = bd.theta.front() >= o.hint_lower && bd.theta.back() <= o.hint_upper;
  }
  if (!hint_used) {
    size_t more = 0;
    bd = lanczos_bounds(op, ops, bound_start, more);
    bound_applications += more;
  }
  // Upper end of the damped interval: the hint's upper end, or the top Ritz
  // value plus its residual norm and 1% of the Ritz range. Components a little
  // above it grow only like exp(d sqrt(2 delta)), far below the amplification
  // of the wanted end.
  const double upper = hint_used ? o.hint_upper
                                 : bd.theta.back() + bd.top_residual + 0.01 * (bd.theta.back() - bd.theta.front());
  double lower = bd.theta.front();
  // First cut: the k-th Ritz value, which lies at or above the k-th eigenvalue.
  // With an accepted hint, the predicted gap places it nb gaps above the
  // interval's lower end when that is lower (the level density grows with
  // energy, so nb gaps lie above the block's share of the spectrum); a cut
  // near the wanted end lets the first filters take a high degree.
  double cut = bd.theta[std::min<size_t>(k, bd.theta.size()) - 1];
  if (hint_used && o.hint_gap > 0.0) cut = std::min(cut, o.hint_lower + nb * o.hint_gap);
  if (!(cut > lower)) cut = lower + 0.1 * (upper - lower);

  std::vector<double> theta, res;
  int iterations[2] = {0, 0};
  bool first_filter = true;
  auto rho = [&](double x, double c, double e) { return std::acosh(std::max((c - x) / e, 1.0)); };

  // One precision phase: filter, orthonormalise, Rayleigh-Ritz until every
  // wanted residual meets target * max(|theta|, 1). Returns whether it did.
  auto phase = [&](int prec, void*& A, void*& B, void* W, double target, int& it) {
    double best = std::numeric_limits<double>::infinity();
    int stall = 0;
    while (true) {
      double worst = 0.0;
      bool done = true;
      for (int i = 0; i < k; ++i) {
        const double scale = std::max(std::fabs(theta[i]), 1.0);
        worst = std::max(worst, res[i] / scale);
        if (!(res[i] <= target * scale)) done = false;
      }
      if (done) return true;
      if (worst < 0.5 * best) {
        best = worst;
        stall = 0;
      } else if (++stall >= 3) {
        return false;
      }
      if (it >= kMaxOuter) return false;
      lower = std::min(lower, theta.front());
      // The first filter of a start block uses the Lanczos (or hinted) cut
      // when it is lower. A random start block's Ritz values all sit near the
      // middle of the spectrum; a hinted cut below them is kept (it only has
      // to stay above the spectrum's lower estimate), every other cut stays
      // above the block's lowest Ritz value.
      const bool hinted_first = first_filter && hint_used && o.hint_gap > 0.0;
      cut = first_filter ? std::min(theta.back(), cut) : theta.back();
      first_filter = false;
      if (!(cut > (hinted_first ? lower : theta.front()))) cut = theta.front() + 1.0e-3 * (upper - theta.front());
      const double e = 0.5 * (upper - cut), c = 0.5 * (upper + cut);
      if (!(e > 0.0)) return false;
      double need = 1.0;
      for (int i = 0; i < k; ++i) {
        const double goal = 0.5 * target * std::max(std::fabs(theta[i]), 1.0);
        if (res[i] > goal) need = std::max(need, std::log(res[i] / goal) / std::max(rho(theta[i], c, e), 1.0e-3));
      }
      const double spread = std::max(rho(lower, c, e), 1.0e-3);
      // The block is orthonormalised through its Gram matrix: the weakest
      // direction keeps accuracy eps * kappa (FP32 data) or eps * kappa^2 (FP64
      // Gram of FP64 data), kappa ~ exp(degree * rho(theta_0)). Cap kappa.
      const double cap = std::log(prec == 64 ? 1.0e6 : 1.0e5) / spread;
      const int degree = static_cast<int>(std::max(2.0, std::min({std::ceil(need), cap, static_cast<double>(kMaxDegree)})));
      const auto t0 = std::chrono::steady_clock::now();
      solver.filter(prec, A, B, degree, lower, cut, upper);
      solver.orthonormalize(prec, A, B, prec == 64 ? 1 : 2);
      solver.rayleigh_ritz(prec, A, B, W, theta, res);
      ++it;
      if (trace) {
        double after = 0.0;
        for (int i = 0; i < k; ++i) after = std::max(after, res[i] / std::max(std::fabs(theta[i]), 1.0));
        std::fprintf(stderr, "[filter] fp%d it=%d degree=%d need=%.1f cap=%.1f lower=%.6f cut=%.6f upper=%.6f "
                     "worst %.3e -> %.3e  %.1f ms\n", prec, it, degree, need, cap, lower, cut, upper, worst, after,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
      }
    }
  };

  void* A64 = ops.workspace(4, block64);
  void* B64 = ops.workspace(5, block64);
  void* W64 = ops.workspace(6, block64);
  stamp("bounds and start columns");
  // A caller's subspace is first judged in FP64 as given: when it already
  // holds the wanted pairs to the FP32 level, the FP32 phase is skipped (and
  // when it meets the tolerance, no filter step runs at all).
  bool fp64_start = false;
  if (used > 0) {
    solver.import_columns(64, cols, A64);
    solver.orthonormalize(64, A64, B64, 2);
    solver.rayleigh_ritz(64, A64, B64, W64, theta, res);
    double worst = 0.0;
    for (int i = 0; i < k; ++i) worst = std::max(worst, res[i] / std::max(std::fabs(theta[i]), 1.0));
    fp64_start = worst <= kFilterHandover;
  }
  if (!fp64_start) {
    // FP32 phase
    void* A = ops.workspace(1, block32);
    void* B = ops.workspace(2, block32);
    void* W = ops.workspace(3, block32);
    solver.import_columns(32, cols, A);
    solver.orthonormalize(32, A, B, 2);
    solver.rayleigh_ritz(32, A, B, W, theta, res);
    stamp("fp32 start block");
    phase(32, A, B, W, std::max(kFilterHandover, o.tolerance), iterations[0]);
    // FP64 phase seeded with the FP32 block
    ops.convert(A, 32, A64, 64, static_cast<uint64_t>(n) * nb);
    stamp("fp32 phase");
    solver.orthonormalize(64, A64, B64, 2);
    solver.rayleigh_ritz(64, A64, B64, W64, theta, res);
    stamp("fp64 start block");
  }
  const bool reached = phase(64, A64, B64, W64, o.tolerance, iterations[1]);
  const size_t total = static_cast<size_t>(iterations[0] + iterations[1]);
  if (!reached) {
    double worst = 0.0;
    for (int i = 0; i < k; ++i) worst = std::max(worst, res[i]);
    raise_nonconvergence(total, worst);
  }
  EigshResult r;
  r.eigenvalues.assign(theta.begin(), theta.begin() + k);
  r.residuals.assign(res.begin(), res.begin() + k);
  r.iterations = total;
  r.fp32_iterations = static_cast<size_t>(iterations[0]);
  r.fp64_iterations = static_cast<size_t>(iterations[1]);
  r.converged = true;
  r.complex_vectors = false;
  if (o.want_vectors) {
    r.vectors.allocate(static_cast<size_t>(n) * k * sizeof(double));
    solver.export_columns(64, A64, k, r.vectors.as<double>());
  }
  ops.sync();
  stamp("export");
  r.operator_applications = solver.applications + bound_applications;
  r.bound_applications = bound_applications;
  r.hint_used = hint_used ? 1 : 0;
  return r;
}

}  // namespace qmbed
