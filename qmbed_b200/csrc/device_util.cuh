// Device helpers: block reductions/scans, sorted-basis search, colex rank.
#pragma once

#include "common.cuh"

namespace qmbed {

constexpr int kBinomStride = 129;  // binomial table is [n][k], n,k <= 128

// 16-byte vector access to rows of row-major blocks (addresses 16-byte aligned).
// load16 reads through the read-only path: only for data no thread of the
// launch writes. load16_rw is the coherent form for rows a launch rewrites.
__device__ __forceinline__ void load16(const float* p, float (&v)[4]) {
  const float4 t = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load16(const double* p, double (&v)[2]) {
  const double2 t = __ldg(reinterpret_cast<const double2*>(p));
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void load16_rw(const float* p, float (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load16_rw(const double* p, double (&v)[2]) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void store16(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store16(double* p, const double (&v)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

__device__ inline uint32_t warp_sum_u32(uint32_t v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block (blockDim.x a multiple of 32, at most 1024).
__device__ inline uint32_t block_reduce_sum_u32(uint32_t v) {
  __shared__ uint32_t partial[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum_u32(v);
  __syncthreads();
  if (lane == 0) partial[warp] = v;
  __syncthreads();
  uint32_t total = 0;
  if (warp == 0) {
    total = lane < static_cast<int>(blockDim.x >> 5) ? partial[lane] : 0u;
    total = warp_sum_u32(total);
  }
  return total;  // valid in thread 0
}

// Exclusive prefix sum over the block in thread order.
__device__ inline uint32_t block_exclusive_scan_u32(uint32_t v) {
  __shared__ uint32_t warp_totals[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inclusive = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t n = __shfl_up_sync(0xffffffffu, inclusive, o);
    if (lane >= o) inclusive += n;
  }
  __syncthreads();
  if (lane == 31) warp_totals[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < static_cast<int>(blockDim.x >> 5) ? warp_totals[lane] : 0u;
    uint32_t inc = t;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t n = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += n;
    }
    warp_totals[lane] = inc - t;
  }
  __syncthreads();
  return warp_totals[warp] + inclusive - v;
}

// Branch-free search of an ascending array of unique states; returns the
// index of `key` or -1 (the lookup of SpinBasis1D::index, mod.rs:1429-1442).
template <typename S>
__host__ __device__ inline int64_t find_sorted(const S* __restrict__ states, uint64_t n, S key) {
  if (n == 0) return -1;
  uint64_t base = 0, len = n;
  while (len > 1) {
    uint64_t half = len >> 1;
    base = (states[base + half] <= key) ? base + half : base;
    len -= half;
  }
  return states[base] == key ? static_cast<int64_t>(base) : -1;
}

// Colex rank of a fixed-weight state, -1 when the weight differs
// (fixed_weight_state_index, reference src/basis/mod.rs:640-659).
template <typename S>
__host__ __device__ inline int64_t colex_rank_checked(S state, int sites, int weight, const uint64_t* __restrict__ binom) {
  if (popcount_state(state) != weight) return -1;
  uint64_t rank = 0;
  int ordinal = 1;
  for (int position = 0; position < sites; ++position) {
    if ((state >> position) & 1) {
      if (position >= ordinal) rank += binom[position * kBinomStride + ordinal];
      ++ordinal;
    }
  }
  return static_cast<int64_t>(rank);
}

}  // namespace qmbed
