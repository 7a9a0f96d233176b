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
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

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

// D_high[t] = sum over terms with mask inside the bits >= tb of c (-1)^popcount(~(t << tb) & mask)
template <typename T>
__global__ void diag_high_table_kernel(int tb, int sites, int nd, const uint64_t* __restrict__ masks,
                                       const double* __restrict__ coefs, T* __restrict__ table) {
  const uint64_t low = (1ull << tb) - 1ull;
  const uint64_t count = 1ull << (sites - tb);
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < count;
       t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t base = t << tb;
    double d = 0.0;
    for (int k = 0; k < nd; ++k)
      if (masks[k] != 0 && (masks[k] & low) == 0) d += (__popcll(~base & masks[k]) & 1) ? -coefs[k] : coefs[k];
    table[t] = static_cast<T>(d);
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

// ---------------------------------------------------------------------------
// Multi-pass action for chains whose vectors exceed the L2 (TMA-staged boxes)
// ---------------------------------------------------------------------------
//
// Pass A applies the diagonal and the flips of the low TB bits to contiguous
// boxes of 2^TB elements and writes the whole epilogue
//   out = alpha (D x + sum_{i < TB} c_i x[s ^ 2^i]) + beta x + gamma p + kappa q.
// Each later pass takes a group of G higher bits [b0, b0 + G): a box holds the
// 2^G elements that differ only in those bits, for a 64-byte run of the lowest
// bits and a batch of the bits above the run, so every flip of the group is a
// read of the box in shared memory; it adds alpha sum_{i in group} c_i x[s ^ 2^i]
// to out. Boxes come in by TMA (cp.async.bulk for pass A, cp.async.bulk.tensor
// for the strided group boxes) into two shared-memory stages, so the next box
// loads while the current one is used. Every wait on a stage's mbarrier is
// bounded: on time-out the block records the failure in `status` and stops.

constexpr int kPassThreads = 512;
constexpr int kBoxBytes = 32 * 1024;
constexpr int kStages = 3;
constexpr unsigned kWaitPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase `parity` of a stage barrier; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (unsigned polls = 0; polls < kWaitPolls; ++polls)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void tensor_load5(void* dst, const CUtensorMap* map, int c1, int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(c1), "r"(0), "r"(0), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

// One pass of the multi-pass action. GROUP = false: pass A over contiguous
// boxes; GROUP = true: the group [b0, b0 + G) from tensor-map boxes.
struct PassArgs {
  int sites, b0, G, bb;  // group pass: box = run (R bits) x batch (bb bits) x group (G bits)
  int nd;
  const uint64_t* masks;
  const double* coefs;
  const void* low_table;
  const void* high_table;  // pass A: the diagonal part of the bits above the box, per box
  const double* xcoef;
  const void* x;
  void* out;
  const void* p;
  const void* q;
  double alpha, beta, gamma, kr, ki;
  int* status;
};

template <typename T, bool CPLX, int TB, int R, bool GROUP>
__global__ void __launch_bounds__(kPassThreads, 2) flip_pass_kernel(const __grid_constant__ CUtensorMap map,
                                                                 const PassArgs a) {
  using E = typename Elem<T, CPLX>::type;
  constexpr int kBox = 1 << TB;
  constexpr int kPer = kBox / kPassThreads;
  static_assert(kBox % kPassThreads == 0, "box elements must divide among the threads");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  E* stage_buf = reinterpret_cast<E*>(smem_raw);
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ T cx[64];
  __shared__ uint64_t cross_mask[kMaxDiagTerms];
  __shared__ T cross_coef[kMaxDiagTerms];
  __shared__ int n_cross;
  __shared__ T d_high;
  __shared__ int abort_flag;
  __shared__ unsigned long long failed_box;
  const int L = a.sites;
  if (threadIdx.x < L) cx[threadIdx.x] = static_cast<T>(a.xcoef[threadIdx.x]);
  const uint64_t low = (1ull << TB) - 1ull;
  if (threadIdx.x == 0) {
    int c = 0;
    if (!GROUP)
      for (int k = 0; k < a.nd; ++k)
        if ((a.masks[k] & low) != 0 && (a.masks[k] & ~low) != 0) {
          cross_mask[c] = a.masks[k];
          cross_coef[c] = static_cast<T>(a.coefs[k]);
          ++c;
        }
    n_cross = c;
    abort_flag = 0;
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint64_t boxes = 1ull << (L - TB);
  const uint64_t mine = boxes > blockIdx.x ? (boxes - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const E* x = static_cast<const E*>(a.x);
  // global index of box position 0 and the box's load coordinates
  const int batch_shift = GROUP ? a.b0 - R - a.bb : 0;  // bits of the batch coordinate above the box's batch
  auto box_id = [&](uint64_t k) { return blockIdx.x + k * gridDim.x; };
  auto issue = [&](uint64_t k) {
    const uint64_t id = box_id(k);
    E* dst = stage_buf + static_cast<size_t>(k % kStages) * kBox;
    mbar_expect_tx(&full[k % kStages], kBox * static_cast<uint32_t>(sizeof(E)));
    if (GROUP) {
      // id = batch block (low b0 - R - bb bits) | above-group index
      const uint64_t blk = id & ((1ull << batch_shift) - 1);
      const uint64_t above = id >> batch_shift;
      tensor_load5(dst, &map, static_cast<int>(blk << a.bb), static_cast<int>(above), &full[k % kStages]);
    } else {
      bulk_load(dst, x + (id << TB), kBox * static_cast<uint32_t>(sizeof(E)), &full[k % kStages]);
    }
  };
  if (threadIdx.x == 0)
    for (uint64_t k = 0; k < mine && k < static_cast<uint64_t>(kStages); ++k) issue(k);
  const T alpha = static_cast<T>(a.alpha), beta = static_cast<T>(a.beta), gamma = static_cast<T>(a.gamma);
  const T kr = static_cast<T>(a.kr), ki = static_cast<T>(a.ki);
  E* out = static_cast<E*>(a.out);
  const E* pv = static_cast<const E*>(a.p);
  const E* qv = static_cast<const E*>(a.q);
  const T* low_table = static_cast<const T*>(a.low_table);
  const int pos_shift = R + a.bb;  // group pass: box position bit of group bit 0
  // flip coefficients of this pass in registers (TB low bits, or the group's bits)
  constexpr int kFlips = GROUP ? TB - R : TB;
  T coef[kFlips];
#pragma unroll
  for (int i = 0; i < kFlips; ++i) coef[i] = GROUP ? (i < a.G ? cx[a.b0 + i] : static_cast<T>(0)) : cx[i];
  for (uint64_t k = 0; k < mine; ++k) {
    const uint64_t id = box_id(k);
    E* box = stage_buf + static_cast<size_t>(k % kStages) * kBox;
    // Global index of each of this thread's elements, and the operands that
    // come from global memory, loaded before the wait on the box so that
    // their latency overlaps the copy.
    uint64_t sidx[kPer];
    E pre0[kPer], pre1[kPer];
    T lowv[kPer];
    if (GROUP) {
      const uint64_t blk = id & ((1ull << batch_shift) - 1);
      const uint64_t above = id >> batch_shift;
      const uint64_t base = (blk << (a.bb + R)) | (above << (a.b0 + a.G));
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int e = threadIdx.x + u * kPassThreads;
        sidx[u] = base | static_cast<uint64_t>(e & ((1 << pos_shift) - 1)) |
                  (static_cast<uint64_t>(e >> pos_shift) << a.b0);
        pre0[u] = out[sidx[u]];
      }
    } else {
      const uint64_t base = id << TB;
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int j = threadIdx.x + u * kPassThreads;
        sidx[u] = base + j;
        lowv[u] = __ldg(low_table + j);
        pre0[u] = pv ? pv[sidx[u]] : zero_elem<E>();
        pre1[u] = qv ? qv[sidx[u]] : zero_elem<E>();
      }
      if (threadIdx.x == 0) d_high = static_cast<const T*>(a.high_table)[id];
    }
    if (threadIdx.x == 0 && !mbar_wait(&full[k % kStages], static_cast<uint32_t>((k / kStages) & 1))) {
      atomicExch(a.status, 1);
      abort_flag = 1;
      failed_box = k;
    }
    __syncthreads();
    if (abort_flag) break;
    if (GROUP) {
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int e = threadIdx.x + u * kPassThreads;
        E acc = zero_elem<E>();
#pragma unroll
        for (int i = 0; i < kFlips; ++i)
          if (i < a.G) acc = scale_add(acc, coef[i], box[e ^ (1 << (pos_shift + i))]);
        out[sidx[u]] = add(pre0[u], scaled(alpha, acc));
      }
    } else {
      const T dh = d_high;
      const int nc = n_cross;
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int j = threadIdx.x + u * kPassThreads;
        const uint64_t s = sidx[u];
        T d = dh + lowv[u];
        for (int c = 0; c < nc; ++c) d += (__popcll(~s & cross_mask[c]) & 1) ? -cross_coef[c] : cross_coef[c];
        const E xs = box[j];
        E acc = scaled(d, xs);
#pragma unroll
        for (int i = 0; i < kFlips; ++i) acc = scale_add(acc, coef[i], box[j ^ (1 << i)]);
        E o = add(scaled(alpha, acc), scaled(beta, xs));
        if (pv) o = add(o, scaled(gamma, pre0[u]));
        if (qv) o = add(o, kappa_times(kr, ki, pre1[u]));
        out[s] = o;
      }
    }
    __syncthreads();  // every thread is done with this stage (and with d_high)
    if (threadIdx.x == 0 && k + kStages < mine) issue(k + kStages);
  }
  // after a time-out, wait (bounded) for the copies still in flight (the box
  // that timed out and the one issued after it) before leaving
  if (threadIdx.x == 0 && abort_flag)
    for (uint64_t k = failed_box; k < mine && k < failed_box + kStages; ++k)
      mbar_wait(&full[k % kStages], static_cast<uint32_t>((k / kStages) & 1));
}

// Self-test of the bounded stage wait: one thread arms an mbarrier for bytes
// that no copy will deliver and waits `polls` times; status receives 1 when
// the wait gave up (the kernel then returns as the passes do).
__global__ void stage_wait_selftest_kernel(unsigned polls, int* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  mbar_expect_tx(&bar, 16);
  bool done = false;
  for (unsigned i = 0; i < polls && !done; ++i) done = mbar_try_wait(&bar, 0);
  *status = done ? 0 : 1;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) raise(QMBED_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
  return fn;
}

// Tensor map of the group boxes over x (4-byte units): d0 the 64-byte run
// (R bits), d1 the bits between the run and the group (box: bb of them),
// d2 / d3 the group's bits (at most 8 per dimension), d4 the bits above.
CUtensorMap group_map(const void* x, int sites, int esize, int r, int b0, int G, int bb) {
  const int g1 = std::min(G, 8), g2 = G - g1;
  const cuuint64_t dims[5] = {static_cast<cuuint64_t>((esize << r) / 4), 1ull << (b0 - r), 1ull << g1, 1ull << g2,
                              1ull << (sites - b0 - G)};
  const cuuint64_t strides[4] = {static_cast<cuuint64_t>(esize) << r, static_cast<cuuint64_t>(esize) << b0,
                                 static_cast<cuuint64_t>(esize) << (b0 + g1), static_cast<cuuint64_t>(esize) << (b0 + G)};
  const cuuint32_t box[5] = {static_cast<cuuint32_t>((esize << r) / 4), 1u << bb, 1u << g1, 1u << g2, 1u};
  const cuuint32_t elem[5] = {1, 1, 1, 1, 1};
  CUtensorMap map;
  const CUresult rc = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 5, const_cast<void*>(x), dims, strides,
                                           box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) raise(QMBED_CUDA_ERROR, "cuTensorMapEncodeTiled failed with code " + std::to_string(rc));
  return map;
}

// Chooses between the one-pass kernel and the multi-pass action: QMBED_FLIP_PASSES=single|multi
// forces one (tests); otherwise vectors beyond 256 MB take the multi-pass action.
bool use_multipass(uint64_t n, int esize, int sites, int tb) {
  if (const char* env = std::getenv("QMBED_FLIP_PASSES")) {
    if (std::strcmp(env, "single") == 0) return false;
    if (std::strcmp(env, "multi") == 0) return sites > tb;
  }
  return sites > tb && n * static_cast<uint64_t>(esize) >= (256ull << 20);
}

}  // namespace

FlipChain::FlipChain(const FlipChainDesc& d) : sites_(d.sites), n_diag_(static_cast<int>(d.z_masks.size())) {
  if (sites_ < 1 || sites_ > 40) raise(QMBED_UNSUPPORTED_BACKEND, "the flip-chain action covers 1 to 40 sites");
  if (n_diag_ > kMaxDiagTerms) raise(QMBED_UNSUPPORTED_BACKEND, "too many diagonal products for the flip-chain action");
  diag_masks_.allocate(std::max(n_diag_, 1) * sizeof(uint64_t));
  diag_coefs_.allocate(std::max(n_diag_, 1) * sizeof(double));
  x_coefs_.allocate(64 * sizeof(double));
  status_.allocate(sizeof(int));
  QMBED_CUDA(cudaMemset(status_.get(), 0, sizeof(int)));
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
  // TMA boxes (cp.async.bulk needs 16-byte aligned sources; tensor maps
  // 16-byte aligned bases): vectors that start elsewhere, such as offset
  // views, take the one-pass kernel
  auto aligned = [](const void* ptr) { return ptr == nullptr || (reinterpret_cast<uintptr_t>(ptr) & 31) == 0; };
  if (aligned(x) && aligned(out) && aligned(p) && aligned(q) &&
      use_multipass(n, esize, sites_, log2_int(kBoxBytes / esize))) {
    apply_multipass(precision, cplx, x, out, p, q, step, stream, sms);
    return;
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

namespace qmbed {

namespace {

template <typename T, bool C, int TB, int R>
void run_passes(int sites, const PassArgs& base, int esize, cudaStream_t stream, int sms) {
  const size_t smem = static_cast<size_t>(kStages) * kBoxBytes;
  auto pass_a = flip_pass_kernel<T, C, TB, R, false>;
  auto pass_g = flip_pass_kernel<T, C, TB, R, true>;
  QMBED_CUDA(cudaFuncSetAttribute(pass_a, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  QMBED_CUDA(cudaFuncSetAttribute(pass_g, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 1;
  QMBED_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass_a, kPassThreads, smem));
  const uint64_t boxes = 1ull << (sites - TB);
  const unsigned grid =
      static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(boxes, static_cast<uint64_t>(sms) * std::max(per_sm, 1))));
  CUtensorMap unused{};
  pass_a<<<grid, kPassThreads, smem, stream>>>(unused, base);
  QMBED_LAUNCH_CHECK();
  for (int b0 = TB; b0 < sites;) {
    const int G = std::min(TB - R, sites - b0);
    PassArgs g = base;
    g.b0 = b0;
    g.G = G;
    g.bb = TB - R - G;
    const CUtensorMap map = group_map(base.x, sites, esize, R, b0, G, g.bb);
    pass_g<<<grid, kPassThreads, smem, stream>>>(map, g);
    QMBED_LAUNCH_CHECK();
    b0 += G;
  }
}

}  // namespace

void FlipChain::apply_multipass(int precision, bool cplx, const void* x, void* out, const void* p, const void* q,
                                const FlipStep& step, cudaStream_t stream, int sms) const {
  if (x == out || (q && q == out)) raise(QMBED_INVALID_OPTIONS, "the flip-chain action cannot write over x or q");
  const int esize = (precision == 64 ? 8 : 4) * (cplx ? 2 : 1);
  const int tb = log2_int(kBoxBytes / esize);
  // the low-bit diagonal table of this box width
  const size_t need = static_cast<size_t>(esize / (cplx ? 2 : 1)) << tb;
  const int slot = precision == 64 ? 0 : 1;
  const size_t high_need = static_cast<size_t>(esize / (cplx ? 2 : 1)) << (sites_ - tb);
  if (pass_table_bytes_[slot] < need || pass_table_tb_[slot] != tb) {
    pass_tables_[slot].allocate(need);
    pass_high_tables_[slot].allocate(high_need);
    pass_table_bytes_[slot] = need;
    pass_table_tb_[slot] = tb;
    const int blocks = static_cast<int>(std::min<uint64_t>(((1ull << tb) + 255) / 256, 1024));
    const int hblocks = static_cast<int>(std::min<uint64_t>(((1ull << (sites_ - tb)) + 255) / 256, 4096));
    if (precision == 64) {
      diag_low_table_kernel<double><<<blocks, 256, 0, stream>>>(tb, n_diag_, diag_masks_.as<uint64_t>(),
                                                                diag_coefs_.as<double>(), pass_tables_[slot].as<double>());
      diag_high_table_kernel<double><<<hblocks, 256, 0, stream>>>(tb, sites_, n_diag_, diag_masks_.as<uint64_t>(),
                                                                  diag_coefs_.as<double>(),
                                                                  pass_high_tables_[slot].as<double>());
    } else {
      diag_low_table_kernel<float><<<blocks, 256, 0, stream>>>(tb, n_diag_, diag_masks_.as<uint64_t>(),
                                                               diag_coefs_.as<double>(), pass_tables_[slot].as<float>());
      diag_high_table_kernel<float><<<hblocks, 256, 0, stream>>>(tb, sites_, n_diag_, diag_masks_.as<uint64_t>(),
                                                                 diag_coefs_.as<double>(),
                                                                 pass_high_tables_[slot].as<float>());
    }
    QMBED_LAUNCH_CHECK();
  }
  PassArgs a{};
  a.sites = sites_;
  a.nd = n_diag_;
  a.masks = diag_masks_.as<uint64_t>();
  a.coefs = diag_coefs_.as<double>();
  a.low_table = pass_tables_[slot].get();
  a.high_table = pass_high_tables_[slot].get();
  a.xcoef = x_coefs_.as<double>();
  a.x = x;
  a.out = out;
  a.p = p;
  a.q = q;
  a.alpha = step.alpha;
  a.beta = step.beta;
  a.gamma = step.gamma;
  a.kr = step.kappa_re;
  a.ki = step.kappa_im;
  a.status = status_.as<int>();
  if (precision == 64) {
    if (cplx) run_passes<double, true, 11, 2>(sites_, a, esize, stream, sms);
    else run_passes<double, false, 12, 3>(sites_, a, esize, stream, sms);
  } else {
    if (cplx) run_passes<float, true, 12, 3>(sites_, a, esize, stream, sms);
    else run_passes<float, false, 13, 4>(sites_, a, esize, stream, sms);
  }
}

void FlipChain::check_status() const {
  int host = 0;
  QMBED_CUDA(cudaMemcpy(&host, status_.get(), sizeof(int), cudaMemcpyDeviceToHost));
  if (host != 0) {
    QMBED_CUDA(cudaMemset(status_.get(), 0, sizeof(int)));
    raise(QMBED_CUDA_ERROR, "a flip-chain pass timed out waiting for its tile copy");
  }
}

}  // namespace qmbed

namespace qmbed {

int flip_stage_wait_selftest(int device) {
  QMBED_CUDA(cudaSetDevice(device));
  DeviceBuffer status(sizeof(int));
  QMBED_CUDA(cudaMemset(status.get(), 0xff, sizeof(int)));
  stage_wait_selftest_kernel<<<1, 32>>>(1u << 10, status.as<int>());
  QMBED_LAUNCH_CHECK();
  int host = -1;
  QMBED_CUDA(cudaMemcpy(&host, status.get(), sizeof(int), cudaMemcpyDeviceToHost));
  return host;
}

}  // namespace qmbed
