// Dense vector kernels for Lanczos / thick restart, reductions and the small
// FP64 Hermitian eigensolver. All reductions accumulate in FP64 through a
// fixed two-stage tree (per-block partials, then an ordered sum), so results
// do not depend on scheduling.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "device_util.cuh"
#include <cstdlib>
#include <string>

#include "krylov.cuh"

namespace qmbed {

bool dense_on_tensor_cores() {
  static const bool on = [] {
    const char* env = std::getenv("QMBED_DENSE");
    return !(env && std::string(env) == "scalar");
  }();
  return on;
}


namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 8;    // columns per pass of the multi-dot
constexpr int kCombine = 4;  // outputs per pass of the combination kernel

template <typename T, bool CPLX>
__device__ inline void load(const T* __restrict__ p, uint64_t i, double& re, double& im) {
  if (CPLX) {
    re = static_cast<double>(p[2 * i]);
    im = static_cast<double>(p[2 * i + 1]);
  } else {
    re = static_cast<double>(p[i]);
    im = 0.0;
  }
}

template <typename T, bool CPLX>
__device__ inline void store(T* __restrict__ p, uint64_t i, double re, double im) {
  if (CPLX) {
    p[2 * i] = static_cast<T>(re);
    p[2 * i + 1] = static_cast<T>(im);
  } else {
    p[i] = static_cast<T>(re);
  }
}

__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Overlaps of a tall FP64 panel with one vector, one warp per column: each
// block stages a slab of `slab` rows of w in shared memory and its warps
// sweep the columns; every lane keeps eight independent loads in flight.
// partials[(j * G + block) * 2 + {0,1}] as for multi_dot_kernel.
constexpr int kMaxSlab = 2048;
template <bool CPLX>
__global__ void __launch_bounds__(kThreads) panel_dot_kernel(const double* __restrict__ A, uint64_t ld, int m,
                                                             const double* __restrict__ w, uint64_t n, int slab,
                                                             double* __restrict__ partials) {
  constexpr int W = CPLX ? 2 : 1;
  extern __shared__ __align__(16) double ws[];
  const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * slab;
  const int rows = static_cast<int>(min(static_cast<uint64_t>(slab), n - r0));
  for (int t = threadIdx.x; t < rows * W; t += blockDim.x) ws[t] = w[r0 * W + t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t G = gridDim.x;
  for (int j = threadIdx.x >> 5; j < m; j += kThreads / 32) {
    const double* q = A + static_cast<uint64_t>(j) * ld * W + r0 * W;
    double sr = 0.0, si = 0.0;
    for (int r = lane; r < rows; r += 32 * 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = r + 32 * u;
        if (k < rows) {
          if (CPLX) {
            const double2 x = reinterpret_cast<const double2*>(q)[k];
            const double2 y = reinterpret_cast<const double2*>(ws)[k];
            sr += x.x * y.x + x.y * y.y;
            si += x.x * y.y - x.y * y.x;
          } else {
            sr += q[k] * ws[k];
          }
        }
      }
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    if (lane == 0) {
      partials[(static_cast<uint64_t>(j) * G + blockIdx.x) * 2] = sr;
      partials[(static_cast<uint64_t>(j) * G + blockIdx.x) * 2 + 1] = si;
    }
  }
}

// partials[(j * G + block) * 2 + {0,1}] = sum over this block's rows of conj(A_j) w.
// With `with_self`, column m receives sum |w|^2 (computed in the first pass).
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kThreads) multi_dot_kernel(const T* __restrict__ A, uint64_t ld, int m,
                                                              const T* __restrict__ w, uint64_t n,
                                                              double* __restrict__ partials, int with_self) {
  __shared__ double red[kThreads / 32][2 * kChunk];
  const int G = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t stride = static_cast<uint64_t>(G) * blockDim.x;
  double self = 0.0;
  for (int j0 = 0; j0 < m; j0 += kChunk) {
    const int cnt = min(kChunk, m - j0);
    double ar[kChunk], ai[kChunk];
#pragma unroll
    for (int jj = 0; jj < kChunk; ++jj) ar[jj] = ai[jj] = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
      double wr, wi;
      load<T, CPLX>(w, i, wr, wi);
      if (j0 == 0) self += wr * wr + wi * wi;
#pragma unroll
      for (int jj = 0; jj < kChunk; ++jj) {
        if (jj < cnt) {
          double xr, xi;
          load<T, CPLX>(A + (j0 + jj) * ld * (CPLX ? 2 : 1), i, xr, xi);
          ar[jj] += xr * wr + xi * wi;
          ai[jj] += xr * wi - xi * wr;
        }
      }
    }
#pragma unroll
    for (int jj = 0; jj < kChunk; ++jj) {
      double a = warp_sum(ar[jj]);
      double b = warp_sum(ai[jj]);
      if (lane == 0) {
        red[warp][2 * jj] = a;
        red[warp][2 * jj + 1] = b;
      }
    }
    __syncthreads();
    if (threadIdx.x < 2 * cnt) {
      double total = 0.0;
      for (int wv = 0; wv < kThreads / 32; ++wv) total += red[wv][threadIdx.x];
      const int j = j0 + threadIdx.x / 2;
      partials[(static_cast<uint64_t>(j) * G + blockIdx.x) * 2 + (threadIdx.x & 1)] = total;
    }
    __syncthreads();
  }
  if (with_self) {
    const double s = warp_sum(self);
    if (lane == 0) red[warp][0] = s;
    __syncthreads();
    if (threadIdx.x < 2) {
      double total = 0.0;
      if (threadIdx.x == 0)
        for (int wv = 0; wv < kThreads / 32; ++wv) total += red[wv][0];
      partials[(static_cast<uint64_t>(m) * G + blockIdx.x) * 2 + threadIdx.x] = total;
    }
  }
}

// out[t] = sum_b partials[(t/2 * G + b) * 2 + t%2]: one block per output,
// strided per-thread sums then a shared-memory tree, both in a fixed order.
constexpr int kFinishThreads = 128;
__global__ void __launch_bounds__(kFinishThreads) finish_kernel(const double* __restrict__ partials, int G, int count,
                                                                double* __restrict__ out) {
  const int t = blockIdx.x;
  if (t >= count) return;
  const int j = t / 2, c = t & 1;
  double total = 0.0;
  for (int b = threadIdx.x; b < G; b += kFinishThreads) total += partials[(static_cast<uint64_t>(j) * G + b) * 2 + c];
  __shared__ double tree[kFinishThreads];
  tree[threadIdx.x] = total;
  __syncthreads();
  for (int width = kFinishThreads / 2; width > 0; width >>= 1) {
    if (threadIdx.x < width) tree[threadIdx.x] += tree[threadIdx.x + width];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[t] = tree[0];
}

// w = src - sum_j h_j A_j (src may be w); per-block partial of ||w||^2 when
// `partials` is set.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kThreads) subtract_kernel(const T* __restrict__ A, uint64_t ld, int m,
                                                             const double* __restrict__ h, const T* src, T* w,
                                                             uint64_t n, double* __restrict__ partials) {
  extern __shared__ double hs[];
  for (int t = threadIdx.x; t < 2 * m; t += blockDim.x) hs[t] = h[t];
  __syncthreads();
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t col = ld * (CPLX ? 2 : 1);
  double sq = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double wr, wi;
    load<T, CPLX>(src, i, wr, wi);
    double sr = 0.0, si = 0.0;
    // batches of kChunk independent loads keep several requests in flight per thread
    for (int j0 = 0; j0 < m; j0 += kChunk) {
      double xr[kChunk], xi[kChunk];
#pragma unroll
      for (int jj = 0; jj < kChunk; ++jj) {
        if (j0 + jj < m) load<T, CPLX>(A + (j0 + jj) * col, i, xr[jj], xi[jj]);
        else xr[jj] = xi[jj] = 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < kChunk; ++jj) {
        if (j0 + jj < m) {
          const double hr = hs[2 * (j0 + jj)], hi = hs[2 * (j0 + jj) + 1];
          sr += hr * xr[jj] - hi * xi[jj];
          si += hr * xi[jj] + hi * xr[jj];
        }
      }
    }
    // norm of the value as stored (rounded to T)
    const T rr = static_cast<T>(wr - sr), ri = static_cast<T>(wi - si);
    store<T, CPLX>(w, i, static_cast<double>(rr), static_cast<double>(ri));
    if (partials) sq += static_cast<double>(rr) * static_cast<double>(rr) + (CPLX ? static_cast<double>(ri) * static_cast<double>(ri) : 0.0);
  }
  if (partials) {
    __shared__ double red[kThreads / 32];
    sq = warp_sum(sq);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double total = 0.0;
      for (int wv = 0; wv < kThreads / 32; ++wv) total += red[wv];
      partials[2 * blockIdx.x] = total;
      partials[2 * blockIdx.x + 1] = 0.0;
    }
  }
}

// out_k = sum_j Y[j + m k] A_j for k in [k0, k0 + kCombine).
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kThreads) combine_kernel(const T* __restrict__ A, uint64_t ld, int m,
                                                            const double* __restrict__ Y, int K, int k0,
                                                            T* __restrict__ out, uint64_t ld_out, uint64_t n) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const int cnt = min(kCombine, K - k0);
  const uint64_t col = ld * (CPLX ? 2 : 1);
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double ar[kCombine], ai[kCombine];
#pragma unroll
    for (int kk = 0; kk < kCombine; ++kk) ar[kk] = ai[kk] = 0.0;
    for (int j0 = 0; j0 < m; j0 += kChunk) {
      double xr[kChunk], xi[kChunk];
#pragma unroll
      for (int jj = 0; jj < kChunk; ++jj) {
        if (j0 + jj < m) load<T, CPLX>(A + (j0 + jj) * col, i, xr[jj], xi[jj]);
        else xr[jj] = xi[jj] = 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < kChunk; ++jj) {
        if (j0 + jj >= m) continue;
#pragma unroll
        for (int kk = 0; kk < kCombine; ++kk) {
          if (kk < cnt) {
            const uint64_t y = (static_cast<uint64_t>(k0 + kk) * m + j0 + jj) * 2;
            const double yr = __ldg(Y + y), yi = __ldg(Y + y + 1);
            ar[kk] += yr * xr[jj] - yi * xi[jj];
            ai[kk] += yr * xi[jj] + yi * xr[jj];
          }
        }
      }
    }
#pragma unroll
    for (int kk = 0; kk < kCombine; ++kk)
      if (kk < cnt) store<T, CPLX>(out + (k0 + kk) * ld_out * (CPLX ? 2 : 1), i, ar[kk], ai[kk]);
  }
}

// Real combinations on the FP64 tensor cores: out[:, k0 + q] = sum_j Re(Y[j, k0 + q]) A[:, j] for
// q < 8, one m8n8k4 DMMA per 8 rows x 4 basis columns. A warp takes tiles of
// 8 consecutive rows; lane l holds A[row 8t + l / 4][column j0 + l % 4] (four
// 64-byte column segments per MMA) and the block's Y columns come from shared
// memory (y[j][q]); D[l / 4][2 (l % 4) + h] is row 8t + l / 4 of output
// column k0 + 2 (l % 4) + h.
template <typename T>
__global__ void __launch_bounds__(kThreads) combine_mma_kernel(const T* __restrict__ A, uint64_t ld, int m,
                                                                const double* __restrict__ Y, int K, int k0,
                                                                T* __restrict__ out, uint64_t ld_out, uint64_t n) {
  extern __shared__ double ys[];  // ys[j * 8 + q] = Re Y[j, k0 + q], zero-padded to a multiple of 4 rows
  const int m4 = (m + 3) & ~3;
  for (int t = threadIdx.x; t < m4 * 8; t += blockDim.x) {
    const int j = t / 8, q = t % 8;
    ys[t] = (j < m && k0 + q < K) ? Y[(static_cast<uint64_t>(k0 + q) * m + j) * 2] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int r = lane >> 2, kq = lane & 3;
  const uint64_t tiles = (n + 7) / 8;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); t < tiles; t += warps) {
    const uint64_t row = t * 8 + r;
    const bool in = row < n;
    double c0 = 0.0, c1 = 0.0;
    for (int j0 = 0; j0 < m4; j0 += 16) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + 4 * u + kq;
        a[u] = (in && j < m) ? static_cast<double>(A[static_cast<uint64_t>(j) * ld + row]) : 0.0;
        b[u] = j < m4 ? ys[j * 8 + r] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(c0), "+d"(c1)
                     : "d"(a[u]), "d"(b[u]));
    }
    const int q0 = k0 + 2 * kq;
    if (in && q0 < K) out[static_cast<uint64_t>(q0) * ld_out + row] = static_cast<T>(c0);
    if (in && q0 + 1 < K) out[static_cast<uint64_t>(q0 + 1) * ld_out + row] = static_cast<T>(c1);
  }
}

template <typename T>
__global__ void scale_kernel(T* __restrict__ w, uint64_t count, double divisor) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
    w[i] = static_cast<T>(static_cast<double>(w[i]) / divisor);
}

template <typename T>
__global__ void scale_into_kernel(const T* __restrict__ src, T* __restrict__ dst, uint64_t count, double divisor) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
    dst[i] = static_cast<T>(static_cast<double>(src[i]) / divisor);
}

__global__ void widen_real_kernel(const double* __restrict__ src, double* __restrict__ dst, uint64_t n) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    dst[2 * i] = src[i];
    dst[2 * i + 1] = 0.0;
  }
}

template <typename D>
__global__ void real_part_strided_kernel(const double* __restrict__ src, D* __restrict__ dst, uint64_t n) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = static_cast<D>(src[2 * i]);
}

template <typename S, typename D>
__global__ void convert_kernel(const S* __restrict__ src, D* __restrict__ dst, uint64_t count) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
    dst[i] = static_cast<D>(src[i]);
}

// Affine LCG state after k steps: x -> a x + c (mod 2^64), by squaring.
__device__ inline uint64_t lcg_jump(uint64_t x, uint64_t k) {
  uint64_t A = 1, C = 0;                                       // accumulated map
  uint64_t a = 6364136223846793005ULL, c = 1442695040888963407ULL;  // current power
  while (k) {
    if (k & 1) {
      A = a * A;
      C = a * C + c;
    }
    c = a * c + c;
    a = a * a;
    k >>= 1;
  }
  return A * x + C;
}

// Element i takes the (i+1)-th LCG state. A block covers blockDim * per_thread
// consecutive elements; thread t takes base + t, base + t + blockDim, ...,
// advancing its state by the blockDim-step map (A, C) between them, so every
// warp store is contiguous.
template <typename T, bool CPLX>
__global__ void lcg_start_kernel(T* __restrict__ out, uint64_t n, uint64_t seed, uint64_t per_thread) {
  const uint64_t stride = blockDim.x;
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * stride * per_thread;
  const uint64_t i0 = base + threadIdx.x;
  if (i0 >= n) return;
  const uint64_t C = lcg_jump(0, stride);
  const uint64_t A = lcg_jump(1, stride) - C;  // the jump is affine: jump(x) = A x + C
  uint64_t state = lcg_jump(seed | 1ULL, i0 + 1);
  const uint64_t end = min(base + stride * per_thread, n);
  for (uint64_t i = i0; i < end; i += stride) {
    const uint64_t mantissa = state >> 11;
    const double value = static_cast<double>(mantissa) / 9007199254740992.0 - 0.5;
    store<T, CPLX>(out, i, value, 0.0);
    state = A * state + C;
  }
}

template <typename T, bool CPLX>
__global__ void __launch_bounds__(kThreads) residual_kernel(const T* __restrict__ y, const T* __restrict__ x,
                                                             double lambda, uint64_t n,
                                                             double* __restrict__ partials) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  double sq = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double yr, yi, xr, xi;
    load<T, CPLX>(y, i, yr, yi);
    load<T, CPLX>(x, i, xr, xi);
    const double dr = yr - lambda * xr, di = yi - lambda * xi;
    sq += dr * dr + di * di;
  }
  __shared__ double red[kThreads / 32];
  sq = warp_sum(sq);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int wv = 0; wv < kThreads / 32; ++wv) total += red[wv];
    partials[2 * blockIdx.x] = total;
    partials[2 * blockIdx.x + 1] = 0.0;
  }
}

// --- scans and reductions used by assembly -------------------------------------------
constexpr int kScanItems = 4;

__global__ void scan_block_totals_kernel(const uint32_t* __restrict__ counts, uint64_t n,
                                         uint64_t* __restrict__ totals) {
  const uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kScanItems;
  uint32_t local = 0;
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) local += counts[base + k];
  uint32_t total = block_reduce_sum_u32(local);
  if (threadIdx.x == 0) totals[blockIdx.x] = total;
}

template <typename IDX>
__global__ void scan_write_kernel(const uint32_t* __restrict__ counts, uint64_t n,
                                  const uint64_t* __restrict__ block_offsets, IDX* __restrict__ out) {
  const uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kScanItems;
  uint32_t local[kScanItems];
  uint32_t sum = 0;
  for (int k = 0; k < kScanItems; ++k) {
    local[k] = base + k < n ? counts[base + k] : 0u;
    sum += local[k];
  }
  uint64_t running = block_offsets[blockIdx.x] + block_exclusive_scan_u32(sum);
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k <= n) out[base + k] = static_cast<IDX>(running);
    running += local[k];
  }
}

__global__ void __launch_bounds__(kThreads) sum_complex_kernel(const double* __restrict__ v, uint64_t n,
                                                                double* __restrict__ partials) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  double re = 0.0, im = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    re += v[2 * i];
    im += v[2 * i + 1];
  }
  __shared__ double red[kThreads / 32][2];
  re = warp_sum(re);
  im = warp_sum(im);
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = re;
    red[threadIdx.x >> 5][1] = im;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double total = 0.0;
    for (int wv = 0; wv < kThreads / 32; ++wv) total += red[wv][threadIdx.x];
    partials[2 * blockIdx.x + threadIdx.x] = total;
  }
}

__global__ void __launch_bounds__(kThreads) max_shifted_kernel(const double* __restrict__ diag,
                                                                const double* __restrict__ offsum, uint64_t n,
                                                                double sr, double si, double* __restrict__ partials) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  double m = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    m = fmax(m, offsum[i] + hypot(diag[2 * i] - sr, diag[2 * i + 1] - si));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int wv = 0; wv < kThreads / 32; ++wv) total = fmax(total, red[wv]);
    partials[blockIdx.x] = total;
  }
}

// --- parallel cyclic Jacobi (one CTA) ---------------------------------------------------
// A: np x np row-major complex (interleaved), V: np x np column-major complex.
// Round-robin ordering pairs np/2 disjoint (p,q) per round; each rotation
// zeroes |a_pq| after removing its phase (complex Jacobi rotation).
__global__ void __launch_bounds__(1024) jacobi_kernel(int np, double* __restrict__ A, double* __restrict__ V,
                                                      int max_sweeps) {
  extern __shared__ int order[];
  __shared__ double c_s[512], s_s[512], pr_s[512], pi_s[512];
  __shared__ int p_s[512], q_s[512];
  __shared__ double red[32][2];
  __shared__ int done;
  __shared__ double previous_off;
  const int half = np / 2;
  // Converged when the off-diagonal mass is at rounding level for this size,
  // or when a sweep no longer reduces it (rounding floor reached).
  const double floor_rel = (2.220446049250313e-16 * np) * (2.220446049250313e-16 * np) * 1e-2;
  if (threadIdx.x == 0) previous_off = -1.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) order[i] = i;
  for (int idx = threadIdx.x; idx < np * np; idx += blockDim.x) {
    V[2 * idx] = (idx / np == idx % np) ? 1.0 : 0.0;
    V[2 * idx + 1] = 0.0;
  }
  __syncthreads();
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0, total = 0.0;
    for (int idx = threadIdx.x; idx < np * np; idx += blockDim.x) {
      const double v = A[2 * idx] * A[2 * idx] + A[2 * idx + 1] * A[2 * idx + 1];
      total += v;
      if (idx / np != idx % np) off += v;
    }
    off = warp_sum(off);
    total = warp_sum(total);
    if ((threadIdx.x & 31) == 0) {
      red[threadIdx.x >> 5][0] = off;
      red[threadIdx.x >> 5][1] = total;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double o = 0.0, t = 0.0;
      for (int wv = 0; wv < static_cast<int>(blockDim.x >> 5); ++wv) {
        o += red[wv][0];
        t += red[wv][1];
      }
      // stagnation counts only once the off-diagonal mass is near rounding level
      const bool stalled = sweep > 4 && previous_off >= 0.0 && o >= 0.5 * previous_off && o <= 1e-24 * t;
      done = (o <= floor_rel * t || o == 0.0 || stalled) ? 1 : 0;
      previous_off = o;
    }
    __syncthreads();
    if (done) break;
    for (int round = 0; round < np - 1; ++round) {
      for (int t = threadIdx.x; t < half; t += blockDim.x) {
        int p = order[t], q = order[np - 1 - t];
        if (p > q) {
          const int tmp = p;
          p = q;
          q = tmp;
        }
        p_s[t] = p;
        q_s[t] = q;
        const double br = A[2 * (p * np + q)], bi = A[2 * (p * np + q) + 1];
        const double mag = hypot(br, bi);
        if (mag == 0.0) {
          c_s[t] = 1.0;
          s_s[t] = 0.0;
          pr_s[t] = 1.0;
          pi_s[t] = 0.0;
        } else {
          const double app = A[2 * (p * np + p)], aqq = A[2 * (q * np + q)];
          const double theta = (aqq - app) / (2.0 * mag);
          const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          const double c = 1.0 / sqrt(tt * tt + 1.0);
          c_s[t] = c;
          s_s[t] = tt * c;
          pr_s[t] = br / mag;
          pi_s[t] = bi / mag;
        }
      }
      __syncthreads();
      // rows: A <- J^H A
      for (int idx = threadIdx.x; idx < half * np; idx += blockDim.x) {
        const int t = idx / np, k = idx % np;
        const int p = p_s[t], q = q_s[t];
        const double c = c_s[t], s = s_s[t], fr = pr_s[t], fi = pi_s[t];
        const double apr = A[2 * (p * np + k)], api = A[2 * (p * np + k) + 1];
        const double aqr = A[2 * (q * np + k)], aqi = A[2 * (q * np + k) + 1];
        // p: c a_p - s phase a_q ; q: s conj(phase) a_p + c a_q
        A[2 * (p * np + k)] = c * apr - s * (fr * aqr - fi * aqi);
        A[2 * (p * np + k) + 1] = c * api - s * (fr * aqi + fi * aqr);
        A[2 * (q * np + k)] = s * (fr * apr + fi * api) + c * aqr;
        A[2 * (q * np + k) + 1] = s * (fr * api - fi * apr) + c * aqi;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J
      for (int idx = threadIdx.x; idx < half * np; idx += blockDim.x) {
        const int t = idx / np, k = idx % np;
        const int p = p_s[t], q = q_s[t];
        const double c = c_s[t], s = s_s[t], fr = pr_s[t], fi = pi_s[t];
        {
          const double apr = A[2 * (k * np + p)], api = A[2 * (k * np + p) + 1];
          const double aqr = A[2 * (k * np + q)], aqi = A[2 * (k * np + q) + 1];
          // p: c a_p - s conj(phase) a_q ; q: s phase a_p + c a_q
          A[2 * (k * np + p)] = c * apr - s * (fr * aqr + fi * aqi);
          A[2 * (k * np + p) + 1] = c * api - s * (fr * aqi - fi * aqr);
          A[2 * (k * np + q)] = s * (fr * apr - fi * api) + c * aqr;
          A[2 * (k * np + q) + 1] = s * (fr * api + fi * apr) + c * aqi;
        }
        {
          const double vpr = V[2 * (p * np + k)], vpi = V[2 * (p * np + k) + 1];
          const double vqr = V[2 * (q * np + k)], vqi = V[2 * (q * np + k) + 1];
          V[2 * (p * np + k)] = c * vpr - s * (fr * vqr + fi * vqi);
          V[2 * (p * np + k) + 1] = c * vpi - s * (fr * vqi - fi * vqr);
          V[2 * (q * np + k)] = s * (fr * vpr - fi * vpi) + c * vqr;
          V[2 * (q * np + k) + 1] = s * (fr * vpi + fi * vpr) + c * vqi;
        }
      }
      __syncthreads();
      for (int t = threadIdx.x; t < half; t += blockDim.x) {
        const int p = p_s[t], q = q_s[t];
        if (c_s[t] != 1.0 || s_s[t] != 0.0) {
          A[2 * (p * np + q)] = A[2 * (p * np + q) + 1] = 0.0;
          A[2 * (q * np + p)] = A[2 * (q * np + p) + 1] = 0.0;
          A[2 * (p * np + p) + 1] = 0.0;
          A[2 * (q * np + q) + 1] = 0.0;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        const int last = order[np - 1];
        for (int i = np - 1; i > 1; --i) order[i] = order[i - 1];
        order[1] = last;
      }
      __syncthreads();
    }
  }
}

int sm_count(int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms;
}

int reduction_grid(uint64_t n, int sms) {
  uint64_t blocks = (n + kThreads - 1) / kThreads;
  return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(blocks, static_cast<uint64_t>(4) * sms)));
}

int stream_grid(uint64_t n, int sms) {
  uint64_t blocks = (n + kThreads - 1) / kThreads;
  return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(blocks, static_cast<uint64_t>(8) * sms)));
}

constexpr int kOrthoThreads = 256;
constexpr int kOrthoChunk = 8;

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < kOrthoThreads / 32; ++k) total += red[k];
  __syncthreads();
  return total;
}

// One Gram-Schmidt pass of the Lanczos step over the basis panel Q (m
// columns, leading dimension n, FP64): w -= sum_k h_k q_k with the overlaps
// h (device, interleaved complex), reading src (which may be w) and writing
// w. Per-block partial sums, in a fixed order: partials[2b] = |w'|^2 for the
// three-term residual w' = src - Re(h_{m-1}) q_{m-1} - beta q_{m-2}
// (before_mode 1) or |src|^2 (before_mode 2), partials[2b+1] =
// |src - sum_k h_k q_k|^2. Elements are complex values
// (kComplex), pairs of real rows loaded as one 16-byte word (kRealPair, n
// even), or single real rows (kReal).
enum { kReal = 0, kRealPair = 1, kComplex = 2 };
template <int MODE>
__global__ void __launch_bounds__(kOrthoThreads, 4) orthogonalize_kernel(const double* __restrict__ Q, uint64_t n, int m,
                                                                      const double* __restrict__ h, double beta,
                                                                      int before_mode, const double* src,
                                                                      double* w, double* __restrict__ partials) {
  extern __shared__ double hs[];
  __shared__ double red[kOrthoThreads / 32];
  for (int t = threadIdx.x; t < 2 * m; t += blockDim.x) hs[t] = h[t];
  __syncthreads();
  const double alpha = hs[2 * (m - 1)];
  // element count and the stride between columns, in elements
  const uint64_t elems = MODE == kRealPair ? n / 2 : n;
  const uint64_t col = MODE == kReal ? n : n / (MODE == kRealPair ? 2 : 1);
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  // columns loaded ahead per element: eight 8-byte or four 16-byte words
  constexpr int CH = MODE == kReal ? kOrthoChunk : kOrthoChunk / 2;
  double before = 0.0, after = 0.0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < elems; i += stride) {
    // (a, b): real and imaginary parts, or the two rows of a pair
    double wa, wb = 0.0;
    if (MODE == kReal) {
      wa = src[i];
    } else {
      const double2 v = reinterpret_cast<const double2*>(src)[i];
      wa = v.x;
      wb = v.y;
    }
    double sa = 0.0, sb = 0.0, la = 0.0, lb = 0.0, pa = 0.0, pb = 0.0;
    for (int j0 = 0; j0 < m; j0 += CH) {
      double xa[CH], xb[CH];
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) {
        xa[jj] = xb[jj] = 0.0;
        if (j0 + jj < m) {
          if (MODE == kReal) {
            xa[jj] = Q[static_cast<uint64_t>(j0 + jj) * col + i];
          } else {
            const double2 v = reinterpret_cast<const double2*>(Q)[static_cast<uint64_t>(j0 + jj) * col + i];
            xa[jj] = v.x;
            xb[jj] = v.y;
          }
        }
      }
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) {
        const int k = j0 + jj;
        if (k < m) {
          const double hr = hs[2 * k], hi = hs[2 * k + 1];
          if (MODE == kComplex) {
            sa += hr * xa[jj] - hi * xb[jj];
            sb += hr * xb[jj] + hi * xa[jj];
          } else {  // real basis: the overlaps are real
            sa += hr * xa[jj];
            sb += hr * xb[jj];
          }
          if (k == m - 1) {
            la = xa[jj];
            lb = xb[jj];
          }
          if (k == m - 2) {
            pa = xa[jj];
            pb = xb[jj];
          }
        }
      }
    }
    if (before_mode == 1) {
      const double ba = wa - alpha * la - beta * pa, bb = wb - alpha * lb - beta * pb;
      before += ba * ba + bb * bb;
    } else if (before_mode == 2) {
      before += wa * wa + wb * wb;
    }
    const double ra = wa - sa, rb = wb - sb;
    if (MODE == kReal) w[i] = ra;
    else reinterpret_cast<double2*>(w)[i] = make_double2(ra, rb);
    after += ra * ra + rb * rb;
  }
  before = block_sum(before, red);
  after = block_sum(after, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = before;
    partials[2 * blockIdx.x + 1] = after;
  }
}

// out[0..1] = sums of the two partial columns over G blocks (fixed order);
// out[2..3] = alpha (the last overlap) for the host's Hermiticity check.
__global__ void __launch_bounds__(128) orthogonalize_finish_kernel(const double* __restrict__ partials, int G,
                                                                   const double* __restrict__ alpha,
                                                                   double* __restrict__ out) {
  __shared__ double tree[2][128];
  double b = 0.0, a = 0.0;
  for (int k = threadIdx.x; k < G; k += 128) {
    b += partials[2 * k];
    a += partials[2 * k + 1];
  }
  tree[0][threadIdx.x] = b;
  tree[1][threadIdx.x] = a;
  __syncthreads();
  for (int width = 64; width > 0; width >>= 1) {
    if (threadIdx.x < width) {
      tree[0][threadIdx.x] += tree[0][threadIdx.x + width];
      tree[1][threadIdx.x] += tree[1][threadIdx.x + width];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = tree[0][0];
    out[1] = tree[1][0];
    out[2] = alpha[0];
    out[3] = alpha[1];
  }
}

}  // namespace

uint64_t exclusive_scan_counts(const uint32_t* counts, uint64_t n, DeviceBuffer& row_ptr, bool* is64) {
  const uint64_t per_block = static_cast<uint64_t>(kThreads) * kScanItems;
  const uint64_t blocks = std::max<uint64_t>(1, (n + 1 + per_block - 1) / per_block);
  DeviceBuffer totals(blocks * sizeof(uint64_t));
  scan_block_totals_kernel<<<static_cast<unsigned>(blocks), kThreads>>>(counts, n, totals.as<uint64_t>());
  QMBED_LAUNCH_CHECK();
  std::vector<uint64_t> host(blocks);
  QMBED_CUDA(cudaMemcpy(host.data(), totals.get(), blocks * 8, cudaMemcpyDeviceToHost));
  uint64_t running = 0;
  for (uint64_t b = 0; b < blocks; ++b) {
    const uint64_t t = host[b];
    host[b] = running;
    running += t;
  }
  QMBED_CUDA(cudaMemcpy(totals.get(), host.data(), blocks * 8, cudaMemcpyHostToDevice));
  *is64 = running >= (1ULL << 32);
  if (*is64) {
    row_ptr.allocate((n + 1) * sizeof(uint64_t));
    scan_write_kernel<uint64_t><<<static_cast<unsigned>(blocks), kThreads>>>(counts, n, totals.as<uint64_t>(),
                                                                            row_ptr.as<uint64_t>());
  } else {
    row_ptr.allocate((n + 1) * sizeof(uint32_t));
    scan_write_kernel<uint32_t><<<static_cast<unsigned>(blocks), kThreads>>>(counts, n, totals.as<uint64_t>(),
                                                                            row_ptr.as<uint32_t>());
  }
  QMBED_LAUNCH_CHECK();
  return running;
}

C64 device_sum_complex(const double* v, uint64_t n) {
  int device = 0;
  cudaGetDevice(&device);
  const int G = reduction_grid(n, sm_count(device));
  DeviceBuffer partials(2 * G * sizeof(double));
  sum_complex_kernel<<<G, kThreads>>>(v, n, partials.as<double>());
  QMBED_LAUNCH_CHECK();
  std::vector<double> host(2 * G);
  QMBED_CUDA(cudaMemcpy(host.data(), partials.get(), host.size() * 8, cudaMemcpyDeviceToHost));
  double re = 0.0, im = 0.0;
  for (int b = 0; b < G; ++b) {
    re += host[2 * b];
    im += host[2 * b + 1];
  }
  return C64(re, im);
}

double device_max_shifted_column(const double* diag, const double* offsum, uint64_t n, C64 shift) {
  int device = 0;
  cudaGetDevice(&device);
  const int G = reduction_grid(n, sm_count(device));
  DeviceBuffer partials(G * sizeof(double));
  max_shifted_kernel<<<G, kThreads>>>(diag, offsum, n, shift.real(), shift.imag(), partials.as<double>());
  QMBED_LAUNCH_CHECK();
  std::vector<double> host(G);
  QMBED_CUDA(cudaMemcpy(host.data(), partials.get(), host.size() * 8, cudaMemcpyDeviceToHost));
  double m = 0.0;
  for (double v : host) m = std::max(m, v);
  return m;
}

BlockOps::BlockOps(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  QMBED_CUDA(cudaSetDevice(device_));
  sms_ = sm_count(device_);
}

BlockOps::~BlockOps() {
  if (host_results_) cudaFreeHost(host_results_);
}

void* BlockOps::workspace(int slot, size_t bytes) {
  if (slot < 0 || slot > 64) raise(QMBED_INTERNAL_STATE, "workspace slot out of range");
  if (workspace_.size() <= static_cast<size_t>(slot)) workspace_.resize(slot + 1);
  DeviceBuffer& b = workspace_[slot];
  if (b.bytes() < bytes) {
    QMBED_CUDA(cudaStreamSynchronize(stream_));  // the old buffer may still be read by queued work
    b.release();
    b.allocate(bytes);
  }
  return b.get();
}

void BlockOps::release_workspace() {
  QMBED_CUDA(cudaStreamSynchronize(stream_));
  workspace_.clear();
}

void BlockOps::ensure_partials(size_t doubles) {
  if (partials_doubles_ < doubles) {
    partials_.allocate(doubles * sizeof(double));
    partials_doubles_ = doubles;
  }
  if (host_results_doubles_ < doubles) {
    if (host_results_) cudaFreeHost(host_results_);
    host_results_ = nullptr;
    QMBED_CUDA(cudaMallocHost(&host_results_, doubles * sizeof(double)));
    host_results_doubles_ = doubles;
    results_.allocate(doubles * sizeof(double));
  }
}

void BlockOps::ensure_coeffs(size_t bytes) {
  if (coeffs_bytes_ < bytes) {
    coeffs_.allocate(bytes);
    coeffs_bytes_ = bytes;
  }
}

void BlockOps::sync() { QMBED_CUDA(cudaStreamSynchronize(stream_)); }

#define QMBED_DISPATCH(precision, cplx, KERNEL_CALL)          \
  do {                                                        \
    if ((precision) == 64) {                                  \
      using T = double;                                       \
      if (cplx) { constexpr bool C = true; KERNEL_CALL; }     \
      else { constexpr bool C = false; KERNEL_CALL; }         \
    } else {                                                  \
      using T = float;                                        \
      if (cplx) { constexpr bool C = true; KERNEL_CALL; }     \
      else { constexpr bool C = false; KERNEL_CALL; }         \
    }                                                         \
  } while (0)

void BlockOps::dots(const void* A, uint64_t ld, int m, const void* w, uint64_t n, int precision, bool cplx,
                    C64* out, double* self_sq) {
  if (m <= 0) {
    if (self_sq) *self_sq = std::pow(norm(w, n, precision, cplx), 2);
    return;
  }
  const int G = reduction_grid(n, sms_);
  const int columns = m + (self_sq ? 1 : 0);
  ensure_partials(static_cast<size_t>(columns) * G * 2 + 2 * static_cast<size_t>(columns) + 64);
  QMBED_DISPATCH(precision, cplx,
                 (multi_dot_kernel<T, C><<<G, kThreads, 0, stream_>>>(static_cast<const T*>(A), ld, m,
                                                                      static_cast<const T*>(w), n,
                                                                      partials_.as<double>(), self_sq ? 1 : 0)));
  QMBED_LAUNCH_CHECK();
  const int count = 2 * columns;
  finish_kernel<<<count, kFinishThreads, 0, stream_>>>(partials_.as<double>(), G, count, results_.as<double>());
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpyAsync(host_results_, results_.get(), count * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
  for (int j = 0; j < m; ++j) out[j] = C64(host_results_[2 * j], host_results_[2 * j + 1]);
  if (self_sq) *self_sq = host_results_[2 * m];
}

void BlockOps::dots_device(const void* A, uint64_t ld, int m, const void* w, uint64_t n, int precision, bool cplx,
                           double* out) {
  if (m <= 0 || n == 0) return;
  int G;
  if (precision == 64) {
    // slabs of 256..2048 rows, sized for about eight blocks per SM
    const uint64_t target = (n + 8ull * sms_ - 1) / (8ull * sms_);
    const int slab = static_cast<int>(std::min<uint64_t>(kMaxSlab, std::max<uint64_t>(256, (target + 255) / 256 * 256)));
    G = static_cast<int>((n + slab - 1) / slab);
    ensure_partials(static_cast<size_t>(m) * G * 2 + 2 * static_cast<size_t>(m) + 64);
    const size_t smem = static_cast<size_t>(slab) * (cplx ? 16 : 8);
    if (cplx)
      panel_dot_kernel<true><<<G, kThreads, smem, stream_>>>(static_cast<const double*>(A), ld, m,
                                                             static_cast<const double*>(w), n, slab,
                                                             partials_.as<double>());
    else
      panel_dot_kernel<false><<<G, kThreads, smem, stream_>>>(static_cast<const double*>(A), ld, m,
                                                              static_cast<const double*>(w), n, slab,
                                                              partials_.as<double>());
  } else {
    G = reduction_grid(n, sms_);
    ensure_partials(static_cast<size_t>(m) * G * 2 + 2 * static_cast<size_t>(m) + 64);
    QMBED_DISPATCH(precision, cplx,
                   (multi_dot_kernel<T, C><<<G, kThreads, 0, stream_>>>(static_cast<const T*>(A), ld, m,
                                                                        static_cast<const T*>(w), n,
                                                                        partials_.as<double>(), 0)));
  }
  QMBED_LAUNCH_CHECK();
  finish_kernel<<<2 * m, kFinishThreads, 0, stream_>>>(partials_.as<double>(), G, 2 * m, out);
  QMBED_LAUNCH_CHECK();
}

void BlockOps::scale_into(const void* src, void* dst, uint64_t n, double divisor, int precision, bool cplx) {
  const uint64_t count = n * (cplx ? 2 : 1);
  const int G = stream_grid(count, sms_);
  if (precision == 64)
    scale_into_kernel<double><<<G, kThreads, 0, stream_>>>(static_cast<const double*>(src), static_cast<double*>(dst),
                                                           count, divisor);
  else
    scale_into_kernel<float><<<G, kThreads, 0, stream_>>>(static_cast<const float*>(src), static_cast<float*>(dst),
                                                          count, divisor);
  QMBED_LAUNCH_CHECK();
}

double BlockOps::norm(const void* w, uint64_t n, int precision, bool cplx) {
  C64 v;
  dots(w, n, 1, w, n, precision, cplx, &v);
  return std::sqrt(std::max(v.real(), 0.0));
}

double BlockOps::subtract(const void* A, uint64_t ld, int m, const C64* h, void* w, uint64_t n, int precision,
                          bool cplx, bool want_norm, const void* src) {
  if (m <= 0 && src && src != w) copy(src, w, n * (cplx ? 2 : 1) * (precision == 64 ? 8 : 4));
  if (m <= 0 && !want_norm) return 0.0;
  if (m <= 0) return norm(w, n, precision, cplx);
  ensure_coeffs(static_cast<size_t>(m) * 16);
  QMBED_CUDA(cudaMemcpyAsync(coeffs_.get(), h, static_cast<size_t>(m) * 16, cudaMemcpyHostToDevice, stream_));
  const int G = reduction_grid(n, sms_);
  ensure_partials(2 * static_cast<size_t>(G) + 64);
  const size_t smem = static_cast<size_t>(m) * 16;
  double* partials = want_norm ? partials_.as<double>() : nullptr;
  QMBED_DISPATCH(precision, cplx, ({
                   auto kernel = subtract_kernel<T, C>;
                   if (smem > 48 * 1024)
                     QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     static_cast<int>(smem)));
                   kernel<<<G, kThreads, smem, stream_>>>(static_cast<const T*>(A), ld, m, coeffs_.as<double>(),
                                                          static_cast<const T*>(src ? src : w), static_cast<T*>(w), n,
                                                          partials);
                 }));
  QMBED_LAUNCH_CHECK();
  if (!want_norm) return 0.0;
  QMBED_CUDA(cudaMemcpyAsync(host_results_, partials_.get(), 2 * G * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
  double total = 0.0;
  for (int b = 0; b < G; ++b) total += host_results_[2 * b];
  return std::sqrt(total);
}

void BlockOps::combine(const void* A, uint64_t ld, int m, const C64* Y, int K, void* out, uint64_t ld_out, uint64_t n,
                       int precision, bool cplx) {
  if (K <= 0) return;
  ensure_coeffs(static_cast<size_t>(m) * K * 16);
  QMBED_CUDA(cudaMemcpyAsync(coeffs_.get(), Y, static_cast<size_t>(m) * K * 16, cudaMemcpyHostToDevice, stream_));
  const int G = stream_grid(n, sms_);
  // real data with real coefficients: the tensor-core kernel, 8 columns per launch
  bool real_y = !cplx;
  for (int i = 0; i < m * K && real_y; ++i) real_y = Y[i].imag() == 0.0;
  const size_t ys_bytes = static_cast<size_t>((m + 3) & ~3) * 8 * sizeof(double);
  if (real_y && dense_on_tensor_cores() && ys_bytes <= 48 * 1024) {
    for (int k0 = 0; k0 < K; k0 += 8) {
      if (precision == 64)
        combine_mma_kernel<double><<<G, kThreads, ys_bytes, stream_>>>(static_cast<const double*>(A), ld, m,
                                                                       coeffs_.as<double>(), K, k0,
                                                                       static_cast<double*>(out), ld_out, n);
      else
        combine_mma_kernel<float><<<G, kThreads, ys_bytes, stream_>>>(static_cast<const float*>(A), ld, m,
                                                                      coeffs_.as<double>(), K, k0,
                                                                      static_cast<float*>(out), ld_out, n);
      QMBED_LAUNCH_CHECK();
    }
    sync();
    return;
  }
  for (int k0 = 0; k0 < K; k0 += kCombine) {
    QMBED_DISPATCH(precision, cplx,
                   (combine_kernel<T, C><<<G, kThreads, 0, stream_>>>(static_cast<const T*>(A), ld, m,
                                                                      coeffs_.as<double>(), K, k0,
                                                                      static_cast<T*>(out), ld_out, n)));
    QMBED_LAUNCH_CHECK();
  }
  sync();  // Y lives in caller memory reused on the next call
}

void BlockOps::scale(void* w, uint64_t n, double divisor, int precision, bool cplx) {
  const uint64_t count = n * (cplx ? 2 : 1);
  const int G = stream_grid(count, sms_);
  if (precision == 64) scale_kernel<double><<<G, kThreads, 0, stream_>>>(static_cast<double*>(w), count, divisor);
  else scale_kernel<float><<<G, kThreads, 0, stream_>>>(static_cast<float*>(w), count, divisor);
  QMBED_LAUNCH_CHECK();
}

void BlockOps::convert(const void* src, int src_precision, void* dst, int dst_precision, uint64_t elements) {
  const int G = stream_grid(elements, sms_);
  if (src_precision == dst_precision) {
    copy(src, dst, elements * (src_precision == 64 ? 8 : 4));
    return;
  }
  if (src_precision == 64)
    convert_kernel<double, float><<<G, kThreads, 0, stream_>>>(static_cast<const double*>(src),
                                                               static_cast<float*>(dst), elements);
  else
    convert_kernel<float, double><<<G, kThreads, 0, stream_>>>(static_cast<const float*>(src),
                                                               static_cast<double*>(dst), elements);
  QMBED_LAUNCH_CHECK();
}

void BlockOps::widen_real(const double* src, double* dst, uint64_t n) {
  const int G = stream_grid(n, sms_);
  widen_real_kernel<<<G, kThreads, 0, stream_>>>(src, dst, n);
  QMBED_LAUNCH_CHECK();
}

void BlockOps::import_complex(const double* src, void* dst, uint64_t n, int precision, bool cplx) {
  if (cplx) {
    convert(src, 64, dst, precision, 2 * n);
    return;
  }
  const int G = stream_grid(n, sms_);
  if (precision == 64) real_part_strided_kernel<double><<<G, kThreads, 0, stream_>>>(src, static_cast<double*>(dst), n);
  else real_part_strided_kernel<float><<<G, kThreads, 0, stream_>>>(src, static_cast<float*>(dst), n);
  QMBED_LAUNCH_CHECK();
}

void BlockOps::copy(const void* src, void* dst, uint64_t bytes) {
  if (bytes == 0 || src == dst) return;
  QMBED_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_));
}

void BlockOps::lcg_start(void* out, uint64_t n, uint64_t seed, int precision, bool cplx) {
  const uint64_t per_thread = 64;
  const uint64_t threads = (n + per_thread - 1) / per_thread;
  const unsigned blocks = static_cast<unsigned>(std::max<uint64_t>(1, (threads + kThreads - 1) / kThreads));
  QMBED_DISPATCH(precision, cplx,
                 (lcg_start_kernel<T, C><<<blocks, kThreads, 0, stream_>>>(static_cast<T*>(out), n, seed,
                                                                           per_thread)));
  QMBED_LAUNCH_CHECK();
}

double BlockOps::residual_norm(const void* y, const void* x, double lambda, uint64_t n, int precision, bool cplx) {
  const int G = reduction_grid(n, sms_);
  ensure_partials(2 * static_cast<size_t>(G) + 64);
  QMBED_DISPATCH(precision, cplx,
                 (residual_kernel<T, C><<<G, kThreads, 0, stream_>>>(static_cast<const T*>(y),
                                                                     static_cast<const T*>(x), lambda, n,
                                                                     partials_.as<double>())));
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpyAsync(host_results_, partials_.get(), 2 * G * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
  double total = 0.0;
  for (int b = 0; b < G; ++b) total += host_results_[2 * b];
  return std::sqrt(total);
}

void device_hermitian_eigen(int n, const std::vector<C64>& a, std::vector<double>& values, std::vector<C64>& vectors,
                            cudaStream_t stream) {
  values.assign(n, 0.0);
  vectors.assign(static_cast<size_t>(n) * n, C64(0.0, 0.0));
  if (n == 0) return;
  if (n == 1) {
    values[0] = a[0].real();
    vectors[0] = C64(1.0, 0.0);
    return;
  }
  if (n > 1024) raise(QMBED_UNSUPPORTED_BACKEND, "projected eigenproblems above 1024 are not supported");
  const int np = n + (n & 1);
  std::vector<double> host(2 * static_cast<size_t>(np) * np, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      host[2 * (static_cast<size_t>(i) * np + j)] = a[static_cast<size_t>(i) * n + j].real();
      host[2 * (static_cast<size_t>(i) * np + j) + 1] = a[static_cast<size_t>(i) * n + j].imag();
    }
  DeviceBuffer dA(host.size() * 8), dV(host.size() * 8);
  QMBED_CUDA(cudaMemcpyAsync(dA.get(), host.data(), host.size() * 8, cudaMemcpyHostToDevice, stream));
  const int threads = std::min(1024, std::max(32, ((np / 2 * np) + 31) / 32 * 32));
  jacobi_kernel<<<1, threads, np * sizeof(int), stream>>>(np, dA.as<double>(), dV.as<double>(), 100);
  QMBED_LAUNCH_CHECK();
  std::vector<double> hv(host.size());
  QMBED_CUDA(cudaMemcpyAsync(host.data(), dA.get(), host.size() * 8, cudaMemcpyDeviceToHost, stream));
  QMBED_CUDA(cudaMemcpyAsync(hv.data(), dV.get(), hv.size() * 8, cudaMemcpyDeviceToHost, stream));
  QMBED_CUDA(cudaStreamSynchronize(stream));
  for (int i = 0; i < n; ++i) values[i] = host[2 * (static_cast<size_t>(i) * np + i)];
  for (int col = 0; col < n; ++col)
    for (int row = 0; row < n; ++row)
      vectors[static_cast<size_t>(col) * n + row] =
          C64(hv[2 * (static_cast<size_t>(col) * np + row)], hv[2 * (static_cast<size_t>(col) * np + row) + 1]);
}

// Ascending eigenpairs of a real symmetric m x m matrix (row-major, symmetrised
// here) on the device; V row-major with eigenvectors as columns.
void device_symmetric_eigen(int m, const std::vector<double>& a, std::vector<double>& values, std::vector<double>& V,
                     cudaStream_t stream) {
  std::vector<C64> ac(static_cast<size_t>(m) * m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) ac[static_cast<size_t>(i) * m + j] = C64(0.5 * (a[i * m + j] + a[j * m + i]), 0.0);
  std::vector<double> vals;
  std::vector<C64> vecs;
  device_hermitian_eigen(m, ac, vals, vecs, stream);
  std::vector<int> order(m);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int l, int r) { return vals[l] < vals[r]; });
  values.assign(m, 0.0);
  V.assign(static_cast<size_t>(m) * m, 0.0);
  for (int q = 0; q < m; ++q) {
    const int col = order[q];
    values[q] = vals[col];
    // eigenvectors of a real matrix are real up to one phase: remove it
    C64 big(0.0, 0.0);
    for (int i = 0; i < m; ++i)
      if (std::abs(vecs[static_cast<size_t>(col) * m + i]) > std::abs(big)) big = vecs[static_cast<size_t>(col) * m + i];
    const C64 phase = std::abs(big) > 0.0 ? std::conj(big) / std::abs(big) : C64(1.0, 0.0);
    for (int i = 0; i < m; ++i) V[static_cast<size_t>(i) * m + q] = (vecs[static_cast<size_t>(col) * m + i] * phase).real();
  }
}


void BlockOps::gram_schmidt_pass(const double* A, uint64_t n, int m, double beta, bool three_term, double* w,
                                 bool cplx, double* before_sq, double* after_sq, C64* last_overlap) {
  if (m <= 0 || n == 0) raise(QMBED_INTERNAL_STATE, "empty Gram-Schmidt pass");
  ensure_coeffs(static_cast<size_t>(m) * 16);
  double* h = coeffs_.as<double>();
  dots_device(A, n, m, w, n, 64, cplx, h);
  const int G = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + kOrthoThreads - 1) / kOrthoThreads,
                                                                          4ull * sms_)));
  ensure_partials(2 * static_cast<size_t>(G) + 64);
  // pairs of real rows move as 16-byte words when every column starts 16-byte aligned
  const int mode = cplx ? kComplex : (n % 2 == 0 ? kRealPair : kReal);
  auto kernel = mode == kComplex ? orthogonalize_kernel<kComplex>
                                 : (mode == kRealPair ? orthogonalize_kernel<kRealPair> : orthogonalize_kernel<kReal>);
  const size_t smem = static_cast<size_t>(m) * 16;
  if (smem > 48 * 1024)
    QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  kernel<<<G, kOrthoThreads, smem, stream_>>>(A, n, m, h, beta, three_term ? 1 : 0, w, w, partials_.as<double>());
  QMBED_LAUNCH_CHECK();
  orthogonalize_finish_kernel<<<1, 128, 0, stream_>>>(partials_.as<double>(), G, h + 2 * (m - 1),
                                                      results_.as<double>());
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpyAsync(host_results_, results_.get(), 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
  *before_sq = host_results_[0];
  *after_sq = host_results_[1];
  if (last_overlap) *last_overlap = C64(host_results_[2], host_results_[3]);
}

void BlockOps::project_out(const double* A, uint64_t n, int m, const double* src, double* w, bool cplx, C64* h,
                           double* src_norm_sq, double* out_norm_sq) {
  if (m <= 0 || n == 0) raise(QMBED_INTERNAL_STATE, "empty projection");
  ensure_coeffs(static_cast<size_t>(m) * 16);
  double* hd = coeffs_.as<double>();
  dots_device(A, n, m, src, n, 64, cplx, hd);
  const int G = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + kOrthoThreads - 1) / kOrthoThreads,
                                                                          4ull * sms_)));
  ensure_partials(2 * static_cast<size_t>(G) + 2 * static_cast<size_t>(m) + 64);
  const int mode = cplx ? kComplex : (n % 2 == 0 ? kRealPair : kReal);
  auto kernel = mode == kComplex ? orthogonalize_kernel<kComplex>
                                 : (mode == kRealPair ? orthogonalize_kernel<kRealPair> : orthogonalize_kernel<kReal>);
  const size_t smem = static_cast<size_t>(m) * 16;
  if (smem > 48 * 1024)
    QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  kernel<<<G, kOrthoThreads, smem, stream_>>>(A, n, m, hd, 0.0, 2, src, w, partials_.as<double>());
  QMBED_LAUNCH_CHECK();
  orthogonalize_finish_kernel<<<1, 128, 0, stream_>>>(partials_.as<double>(), G, hd, results_.as<double>());
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpyAsync(host_results_, results_.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  QMBED_CUDA(cudaMemcpyAsync(host_results_ + 2, hd, static_cast<size_t>(m) * 16, cudaMemcpyDeviceToHost, stream_));
  sync();
  *src_norm_sq = host_results_[0];
  *out_norm_sq = host_results_[1];
  for (int j = 0; j < m; ++j) h[j] = C64(host_results_[2 + 2 * j], host_results_[3 + 2 * j]);
}

// Symmetric tridiagonal eigenproblem (diagonal d, off-diagonal e) by the
// implicit QL method with Wilkinson shifts (Bowdler, Martin, Reinsch and
// Wilkinson, Numer. Math. 11 (1968) 293-306). Rotations are accumulated into
// Z (row-major n x n, Z[k * n + c]) or, with `first_row`, into its first
// row only (all that Boltzmann weights and spectral measures need). Returns ascending values
// with the columns permuted alike.
void tridiagonal_eigen(std::vector<double> d, std::vector<double> e, bool first_row, std::vector<double>& values,
                       std::vector<double>& V) {
  const int n = static_cast<int>(d.size());
  const int rows = first_row ? 1 : n;
  std::vector<double> Z(static_cast<size_t>(rows) * n, 0.0);
  for (int k = 0; k < rows; ++k) Z[static_cast<size_t>(k) * n + k] = 1.0;
  e.resize(static_cast<size_t>(n), 0.0);
  for (int l = 0; l < n; ++l) {
    for (int sweep = 0;; ++sweep) {
      int m = l;
      for (; m + 1 < n; ++m)
        if (std::fabs(e[m]) <= 2.220446049250313e-16 * (std::fabs(d[m]) + std::fabs(d[m + 1]))) break;
      if (m == l) break;
      if (sweep == 60) raise(QMBED_INTERNAL_STATE, "tridiagonal eigensolver did not converge");
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool deflated = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // underflow: split the matrix here and restart
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < rows; ++k) {
          double* z = Z.data() + static_cast<size_t>(k) * n;
          const double t = z[i + 1];
          z[i + 1] = s * z[i] + c * t;
          z[i] = c * z[i] - s * t;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  std::vector<int> order(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
  values.resize(static_cast<size_t>(n));
  V.assign(static_cast<size_t>(rows) * n, 0.0);
  for (int c = 0; c < n; ++c) {
    values[c] = d[order[c]];
    for (int k = 0; k < rows; ++k) V[static_cast<size_t>(k) * n + c] = Z[static_cast<size_t>(k) * n + order[c]];
  }
}


}  // namespace qmbed
