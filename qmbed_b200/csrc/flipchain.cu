// Structured full-space chain action (diagonal z products + single bit flips).
//
// The action is y[s] = D(s) x[s] + sum_i c_i x[s ^ (1 << i)], computed in one
// pass over tiles of 2^tb consecutive elements (64 KB) held in shared memory:
// the flips of the low tb bits read the tile, the flips of the higher bits
// read their partner element from global memory. A partner of bit i lies in
// tile t ^ 2^(i - tb), a contiguous chunk, so those reads are fully coalesced,
// and partner tiles within the L2 window (about 1900 tiles of 64 KB) are
// served by L2. The fused epilogue out = alpha y + beta x + gamma p + kappa q
// serves the Chebyshev (Clenshaw) step.
// D(s) = D_low(j) + D_high(t) + D_cross(s): terms inside the low bits come from
// a 2^tb table computed once, terms inside the high bits once per tile, and
// only the terms spanning both are evaluated per element.
#include <algorithm>
#include <cmath>

#include "device_util.cuh"
#include "flipchain.cuh"

namespace qmbed {

namespace {

constexpr int kTileBytes = 64 * 1024;
constexpr int kFlipThreads = 512;
constexpr int kMaxDiagTerms = 256;

template <typename T, bool CPLX>
struct Elem;
template <typename T>
struct Elem<T, false> {
  using type = T;
};
template <>
struct Elem<float, true> {
  using type = float2;
};
template <>
struct Elem<double, true> {
  using type = double2;
};

template <typename T>
__device__ __forceinline__ T scale_add(T acc, T c, T v) { return acc + c * v; }
__device__ __forceinline__ float2 scale_add(float2 acc, float c, float2 v) {
  return make_float2(acc.x + c * v.x, acc.y + c * v.y);
}
__device__ __forceinline__ double2 scale_add(double2 acc, double c, double2 v) {
  return make_double2(acc.x + c * v.x, acc.y + c * v.y);
}
template <typename T>
__device__ __forceinline__ T scaled(T c, T v) { return c * v; }
__device__ __forceinline__ float2 scaled(float c, float2 v) { return make_float2(c * v.x, c * v.y); }
__device__ __forceinline__ double2 scaled(double c, double2 v) { return make_double2(c * v.x, c * v.y); }
template <typename T>
__device__ __forceinline__ T zero_elem() { return T(0); }
template <>
__device__ __forceinline__ float2 zero_elem<float2>() { return make_float2(0.f, 0.f); }
template <>
__device__ __forceinline__ double2 zero_elem<double2>() { return make_double2(0.0, 0.0); }
// kappa * q with complex kappa (real vectors use its real part)
template <typename T>
__device__ __forceinline__ T kappa_times(T kr, T, T q) { return kr * q; }
__device__ __forceinline__ float2 kappa_times(float kr, float ki, float2 q) {
  return make_float2(kr * q.x - ki * q.y, kr * q.y + ki * q.x);
}
__device__ __forceinline__ double2 kappa_times(double kr, double ki, double2 q) {
  return make_double2(kr * q.x - ki * q.y, kr * q.y + ki * q.x);
}
template <typename T>
__device__ __forceinline__ T add(T a, T b) { return a + b; }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

template <typename E, typename T>
__device__ __forceinline__ E epilogue(E hx, E x, const E* p, const E* q, uint64_t s, T alpha, T beta, T gamma, T kr,
                                      T ki) {
  E o = add(scaled(alpha, hx), scaled(beta, x));
  if (p) o = add(o, scaled(gamma, p[s]));
  if (q) o = add(o, kappa_times(kr, ki, q[s]));
  return o;
}

// D_low[j] = sum over terms with mask inside the low tb bits of c (-1)^popcount(~j & mask)
template <typename T>
__global__ void diag_low_table_kernel(int tb, int nd, const uint64_t* __restrict__ masks,
                                      const double* __restrict__ coefs, T* __restrict__ table) {
  const uint64_t low = (1ull << tb) - 1ull;
  for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < (1ull << tb);
       j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    double d = 0.0;
    for (int k = 0; k < nd; ++k)
      if ((masks[k] & ~low) == 0) d += (__popcll(~j & masks[k]) & 1) ? -coefs[k] : coefs[k];
    table[j] = static_cast<T>(d);
  }
}

// One pass: tile flips, global-partner flips, diagonal and the epilogue.
// TB > 0 fixes the tile bits at compile time (the tile loop unrolls); TB = 0
// takes them from `tb` (chains shorter than a tile).
template <typename T, bool CPLX, int TB>
__global__ void __launch_bounds__(kFlipThreads) flip_chain_kernel(int sites, int tb, int nd,
                                                                const uint64_t* __restrict__ masks,
                                                                const double* __restrict__ coefs,
                                                                const T* __restrict__ low_table,
                                                                const double* __restrict__ xcoef,
                                                                const typename Elem<T, CPLX>::type* __restrict__ x,
                                                                typename Elem<T, CPLX>::type* out,
                                                                const typename Elem<T, CPLX>::type* p,
                                                                const typename Elem<T, CPLX>::type* q, T alpha, T beta,
                                                                T gamma, T kr, T ki) {
  using E = typename Elem<T, CPLX>::type;
  extern __shared__ unsigned char smem_raw[];
  E* tile = reinterpret_cast<E*>(smem_raw);
  __shared__ T cx[64];
  __shared__ uint64_t cross_mask[kMaxDiagTerms];
  __shared__ T cross_coef[kMaxDiagTerms];
  __shared__ int n_cross;
  __shared__ T d_high;
  const uint64_t low = (1ull << tb) - 1ull;
  if (threadIdx.x < sites) cx[threadIdx.x] = static_cast<T>(xcoef[threadIdx.x]);
  if (threadIdx.x == 0) {
    int c = 0;
    for (int k = 0; k < nd; ++k)
      if ((masks[k] & low) != 0 && (masks[k] & ~low) != 0) {
        cross_mask[c] = masks[k];
        cross_coef[c] = static_cast<T>(coefs[k]);
        ++c;
      }
    n_cross = c;
  }
  const uint64_t tiles = 1ull << (sites - tb);
  const int count = 1 << tb;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t base = t << tb;
    __syncthreads();  // previous tile consumed; cross terms ready
    if (threadIdx.x == 0) {
      double d = 0.0;
      for (int k = 0; k < nd; ++k)  // constant terms (mask 0) are in the low table
        if (masks[k] != 0 && (masks[k] & low) == 0) d += (__popcll(~base & masks[k]) & 1) ? -coefs[k] : coefs[k];
      d_high = static_cast<T>(d);
    }
    for (int j = threadIdx.x; j < count; j += blockDim.x) tile[j] = x[base + j];
    __syncthreads();
    const T dh = d_high;
    const int nc = n_cross;
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
      const uint64_t s = base + j;
      T d = dh + __ldg(low_table + j);
      for (int k = 0; k < nc; ++k) d += (__popcll(~s & cross_mask[k]) & 1) ? -cross_coef[k] : cross_coef[k];
      const E xs = tile[j];
      E acc = scaled(d, xs);
      if (TB > 0) {
#pragma unroll
        for (int i = 0; i < TB; ++i) acc = scale_add(acc, cx[i], tile[j ^ (1 << i)]);
      } else {
        for (int i = 0; i < tb; ++i) acc = scale_add(acc, cx[i], tile[j ^ (1 << i)]);
      }
      // high bits: partner elements from global memory, four loads in flight per thread
      int i = TB > 0 ? TB : tb;
      for (; i + 4 <= sites; i += 4) {
        const E y0 = x[s ^ (1ull << i)], y1 = x[s ^ (1ull << (i + 1))];
        const E y2 = x[s ^ (1ull << (i + 2))], y3 = x[s ^ (1ull << (i + 3))];
        acc = scale_add(acc, cx[i], y0);
        acc = scale_add(acc, cx[i + 1], y1);
        acc = scale_add(acc, cx[i + 2], y2);
        acc = scale_add(acc, cx[i + 3], y3);
      }
      for (; i < sites; ++i) acc = scale_add(acc, cx[i], x[s ^ (1ull << i)]);
      out[s] = epilogue(acc, xs, p, q, s, alpha, beta, gamma, kr, ki);
    }
  }
}

int log2_int(int v) {
  int r = 0;
  while ((1 << (r + 1)) <= v) ++r;
  return r;
}

}  // namespace

FlipChain::FlipChain(const FlipChainDesc& d) : sites_(d.sites), n_diag_(static_cast<int>(d.z_masks.size())) {
  if (sites_ < 1 || sites_ > 40) raise(QMBED_UNSUPPORTED_BACKEND, "the flip-chain action covers 1 to 40 sites");
  if (n_diag_ > kMaxDiagTerms) raise(QMBED_UNSUPPORTED_BACKEND, "too many diagonal products for the flip-chain action");
  diag_masks_.allocate(std::max(n_diag_, 1) * sizeof(uint64_t));
  diag_coefs_.allocate(std::max(n_diag_, 1) * sizeof(double));
  x_coefs_.allocate(64 * sizeof(double));
  std::vector<double> x(64, 0.0);
  for (int i = 0; i < sites_; ++i) x[i] = d.x_coefs[i];
  if (n_diag_ > 0) {
    QMBED_CUDA(cudaMemcpy(diag_masks_.get(), d.z_masks.data(), n_diag_ * sizeof(uint64_t), cudaMemcpyHostToDevice));
    QMBED_CUDA(cudaMemcpy(diag_coefs_.get(), d.z_coefs.data(), n_diag_ * sizeof(double), cudaMemcpyHostToDevice));
  }
  QMBED_CUDA(cudaMemcpy(x_coefs_.get(), x.data(), 64 * sizeof(double), cudaMemcpyHostToDevice));
  host_diag_coefs_ = d.z_coefs;
  host_x_ = x;
}

double FlipChain::norm_bound() const {
  double b = 0.0;
  for (double c : host_diag_coefs_) b += std::fabs(c);
  for (double c : host_x_) b += std::fabs(c);
  return b;
}

void FlipChain::apply(int precision, bool cplx, const void* x, void* out, const void* p, const void* q,
                      const FlipStep& step, cudaStream_t stream) const {
  const int esize = (precision == 64 ? 8 : 4) * (cplx ? 2 : 1);
  const int tbits = log2_int(kTileBytes / esize);
  const int tb = std::min(sites_, tbits);
  const uint64_t n = dim();
  int device = 0, sms = 148;
  QMBED_CUDA(cudaGetDevice(&device));
  QMBED_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  // low-bit diagonal tables (2^tb values of the working precision, at most
  // kTileBytes each): FP64 table first, FP32 table second
  const size_t need = 2 * static_cast<size_t>(kTileBytes);
  if (tables_bytes_ < need) {
    tables_.allocate(need);
    tables_bytes_ = need;
    tables_ready_ = 0;
  }
  const int table_slot = precision == 64 ? 1 : 2;
  void* table = static_cast<unsigned char*>(tables_.get()) + (precision == 64 ? 0 : kTileBytes);
  if (!(tables_ready_ & table_slot) || table_tb_[table_slot - 1] != tb) {
    const int blocks = static_cast<int>(std::min<uint64_t>(((1ull << tb) + 255) / 256, 1024));
    if (precision == 64)
      diag_low_table_kernel<double><<<blocks, 256, 0, stream>>>(tb, n_diag_, diag_masks_.as<uint64_t>(),
                                                                diag_coefs_.as<double>(), static_cast<double*>(table));
    else
      diag_low_table_kernel<float><<<blocks, 256, 0, stream>>>(tb, n_diag_, diag_masks_.as<uint64_t>(),
                                                               diag_coefs_.as<double>(), static_cast<float*>(table));
    QMBED_LAUNCH_CHECK();
    tables_ready_ |= table_slot;
    table_tb_[table_slot - 1] = tb;
  }
  const size_t smem = static_cast<size_t>(esize) << tb;
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(n >> tb, 3ull * sms)));
  auto run = [&](auto ttag, auto ctag) {
    using T = decltype(ttag);
    constexpr bool C = decltype(ctag)::value;
    using E = typename Elem<T, C>::type;
    const T a = static_cast<T>(step.alpha), b = static_cast<T>(step.beta), g = static_cast<T>(step.gamma),
            kr = static_cast<T>(step.kappa_re), ki = static_cast<T>(step.kappa_im);
    // the full-tile width for this element size, known at compile time
    constexpr int kFull = (sizeof(E) == 4) ? 14 : (sizeof(E) == 8 ? 13 : 12);
    auto kernel = tb == kFull ? flip_chain_kernel<T, C, kFull> : flip_chain_kernel<T, C, 0>;
    QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kernel<<<grid, kFlipThreads, smem, stream>>>(sites_, tb, n_diag_, diag_masks_.as<uint64_t>(),
                                                 diag_coefs_.as<double>(), static_cast<const T*>(table),
                                                 x_coefs_.as<double>(), static_cast<const E*>(x), static_cast<E*>(out),
                                                 static_cast<const E*>(p), static_cast<const E*>(q), a, b, g, kr, ki);
    QMBED_LAUNCH_CHECK();
  };
  if (precision == 64) cplx ? run(double{}, std::true_type{}) : run(double{}, std::false_type{});
  else cplx ? run(float{}, std::true_type{}) : run(float{}, std::false_type{});
}

}  // namespace qmbed
