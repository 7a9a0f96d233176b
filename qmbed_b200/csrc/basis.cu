// Sector enumeration on the GPU (kernel K1) and the host-side basis object.
//
// Reference behaviour (matrixlab-research/QMBED):
//   fixed_weight_states  src/basis/mod.rs:373-424  (Gosper, colex = numeric order)
//   spin_symmetry_sector src/basis/mod.rs:715-848  (rep = orbit minimum, sorted)
//   SpinBasisBuilder::build src/basis/mod.rs:1312-1412
// The reference hashes every parent state; here each thread walks a colex
// rank range with Gosper's step, keeps states that are their own orbit
// minimum and whose one-dimensional projection is nonzero, and a two-pass
// compaction writes them in rank order, which is ascending numeric order.
#include <chrono>
#include <cmath>
#include <numeric>

#include "basis.cuh"
#include "device_util.cuh"

namespace qmbed {

void DeviceBuffer::allocate(size_t bytes) {
  release();
  if (bytes == 0) return;
  cudaError_t status = cudaMalloc(&ptr_, bytes);
  if (status != cudaSuccess) {
    ptr_ = nullptr;
    (void)cudaGetLastError();
    raise(QMBED_UNSUPPORTED_BACKEND, "device allocation of " + std::to_string(bytes) +
                                         " bytes failed: " + cudaGetErrorString(status));
  }
  bytes_ = bytes;
}

void DeviceBuffer::release() {
  if (ptr_) cudaFree(ptr_);
  ptr_ = nullptr;
  bytes_ = 0;
}

namespace {

constexpr int kEnumThreads = 256;
constexpr uint64_t kEnumChunk = 128;  // ranks per thread; counts fit in u8

template <typename S>
__device__ inline int ctz_state(S v);
template <>
__device__ inline int ctz_state<uint64_t>(uint64_t v) { return __ffsll(static_cast<long long>(v)) - 1; }
template <>
__device__ inline int ctz_state<u128>(u128 v) {
  uint64_t lo = static_cast<uint64_t>(v);
  if (lo) return __ffsll(static_cast<long long>(lo)) - 1;
  return 64 + __ffsll(static_cast<long long>(static_cast<uint64_t>(v >> 64))) - 1;
}

// Colex unrank: the state of weight `weight` at position `rank` of the
// Gosper sequence (combinatorial number system).
template <typename S>
__device__ inline S colex_unrank(uint64_t rank, int sites, int weight, const uint64_t* binom) {
  S state = 0;
  int p = sites - 1;
  for (int i = weight; i >= 1; --i) {
    while (binom[p * kBinomStride + i] > rank) --p;
    state |= static_cast<S>(1) << p;
    rank -= binom[p * kBinomStride + i];
    --p;
  }
  return state;
}

// Gosper's step to the next state of equal weight (reference mod.rs:413-421).
template <typename S>
__device__ inline S gosper_next(S s) {
  S low = s & (~s + 1);
  S ripple = s + low;
  return ripple | (((ripple ^ s) >> 2) >> ctz_state(s));
}

// True when `s` is the minimum of its translation/reflection orbit. Exits at
// the first smaller image, so non-representatives cost a few rotations.
template <typename S>
__device__ inline bool is_orbit_minimum(S s, const SectorParams& p, S mask) {
  const int translations = p.has_momentum ? p.sites : 1;
  for (int sh = 1; sh < translations; ++sh)
    if (rotate_state(s, sh, p.sites, mask) < s) return false;
  if (p.parity != 0) {
    S u = reflect_state(s, p.sites);
    for (int sh = 0; sh < translations; ++sh)
      if (rotate_state(u, sh, p.sites, mask) < s) return false;
  }
  if (p.inversion != 0) {
    const S c = static_cast<S>(~s & mask);
    for (int sh = 0; sh < translations; ++sh)
      if (rotate_state(c, sh, p.sites, mask) < s) return false;
    if (p.parity != 0) {
      S u = reflect_state(c, p.sites);
      for (int sh = 0; sh < translations; ++sh)
        if (rotate_state(u, sh, p.sites, mask) < s) return false;
    }
  }
  return true;
}

template <typename S>
__device__ inline int accept_state(S s, const SectorParams& p, S mask) {
  if (!p.symmetric) return 1;
  if (!is_orbit_minimum(s, p, mask)) return 0;
  return orbit_size_if_compatible(s, p, mask);
}

template <typename S>
__device__ inline S first_state(uint64_t rank, const SectorParams& p, const uint64_t* binom) {
  return p.up >= 0 ? colex_unrank<S>(rank, p.sites, p.up, binom) : static_cast<S>(rank);
}

template <typename S>
__device__ inline S next_state(S s, const SectorParams& p) {
  return p.up >= 0 ? gosper_next(s) : s + 1;
}

template <typename S>
__global__ void enumerate_count_kernel(SectorParams p, uint64_t total, const uint64_t* binom, uint8_t* counts,
                                       uint32_t* block_totals) {
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t r0 = tid * kEnumChunk;
  const S mask = low_mask<S>(p.sites);
  uint32_t count = 0;
  if (r0 < total) {
    const uint64_t r1 = min(r0 + kEnumChunk, total);
    S s = first_state<S>(r0, p, binom);
    for (uint64_t r = r0; r < r1; ++r) {
      count += accept_state(s, p, mask) > 0 ? 1u : 0u;
      if (r + 1 < r1) s = next_state(s, p);
    }
    counts[tid] = static_cast<uint8_t>(count);
  }
  uint32_t block_sum = block_reduce_sum_u32(count);
  if (threadIdx.x == 0) block_totals[blockIdx.x] = block_sum;
}

template <typename S>
__global__ void enumerate_fill_kernel(SectorParams p, uint64_t total, const uint64_t* binom, const uint8_t* counts,
                                      const uint64_t* block_offsets, S* states, uint16_t* orbits) {
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t r0 = tid * kEnumChunk;
  const S mask = low_mask<S>(p.sites);
  uint32_t count = r0 < total ? counts[tid] : 0u;
  uint32_t prefix = block_exclusive_scan_u32(count);
  if (r0 >= total || count == 0) return;
  uint64_t out = block_offsets[blockIdx.x] + prefix;
  const uint64_t r1 = min(r0 + kEnumChunk, total);
  S s = first_state<S>(r0, p, binom);
  for (uint64_t r = r0; r < r1; ++r) {
    int orbit = accept_state(s, p, mask);
    if (orbit > 0) {
      states[out] = s;
      if (orbits) orbits[out] = static_cast<uint16_t>(orbit);
      ++out;
    }
    if (r + 1 < r1) s = next_state(s, p);
  }
}

template <typename S>
__global__ void images_kernel(SectorParams p, const S* states, const uint16_t* orbits, uint64_t dim, int direct,
                              int colex, const uint64_t* binom, const double* phase_table, const uint64_t* lo,
                              const uint64_t* hi, uint64_t n, int64_t* index, double* phase, uint16_t* orbit_out) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  S t = static_cast<S>(lo[i]);
  if (sizeof(S) > 8) t |= static_cast<S>(hi[i]) << 32 << 32;
  const S mask = low_mask<S>(p.sites);
  int64_t idx = -1;
  double pr = 1.0, pi = 0.0;
  uint16_t orbit = 1;
  if ((t & ~mask) == 0) {
    if (direct) {
      idx = static_cast<uint64_t>(t) < dim ? static_cast<int64_t>(t) : -1;
    } else if (colex) {
      idx = colex_rank_checked(t, p.sites, p.up, binom);
    } else {
      Canonical<S> c = canonicalize(t, p, mask);
      idx = find_sorted(states, dim, c.rep);
      if (idx >= 0 && p.symmetric) {
        pr = phase_table[2 * c.shift];
        pi = phase_table[2 * c.shift + 1];
        if (c.reflected) { pr *= p.parity; pi *= p.parity; }
        if (c.inverted) { pr *= p.inversion; pi *= p.inversion; }
        orbit = orbits[idx];
      }
    }
  }
  index[i] = idx;
  phase[2 * i] = idx >= 0 ? pr : 0.0;
  phase[2 * i + 1] = idx >= 0 ? pi : 0.0;
  orbit_out[i] = idx >= 0 ? orbit : 0;
}

uint64_t saturating_binomial(int n, int k) {
  if (k < 0 || k > n) return 0;
  k = std::min(k, n - k);
  unsigned __int128 value = 1;
  for (int i = 0; i < k; ++i) {
    value = value * static_cast<unsigned>(n - i) / static_cast<unsigned>(i + 1);
    if (value > static_cast<unsigned __int128>(UINT64_MAX)) return UINT64_MAX;
  }
  return static_cast<uint64_t>(value);
}

}  // namespace

SpinBasis::SpinBasis(const SpinBasisDesc& desc, int device) : device_(device), normalization_(desc.normalization) {
  auto start = std::chrono::steady_clock::now();
  if (desc.sites <= 0) raise(QMBED_INVALID_SECTOR, "symmetry sectors require at least one site");
  if (desc.sites > kMaxSites)
    raise(QMBED_UNSUPPORTED_BACKEND, "the initial u128 state backend supports at most 128 orbitals");
  if (desc.normalization < 0 || desc.normalization > 2) raise(QMBED_INVALID_OPTIONS, "unknown spin normalization");
  if (desc.up >= 0 && desc.up > desc.sites) raise(QMBED_INVALID_SECTOR, "particle count exceeds site count");
  if (desc.parity != 0 && desc.parity != 1 && desc.parity != -1)
    raise(QMBED_INVALID_SECTOR, "parity must be either -1 or +1");
  SectorParams& p = params_;
  p.sites = desc.sites;
  p.up = desc.up;
  p.has_momentum = desc.has_momentum ? 1 : 0;
  p.momentum = p.has_momentum ? ((desc.momentum % desc.sites) + desc.sites) % desc.sites : 0;
  p.parity = desc.parity;
  if (desc.inversion != 0 && desc.inversion != 1 && desc.inversion != -1)
    raise(QMBED_INVALID_SECTOR, "spin inversion must be either -1 or +1");
  if (desc.inversion != 0 && desc.up >= 0 && 2 * desc.up != desc.sites)
    raise(QMBED_UNSUPPORTED_BACKEND, "spin inversion of a magnetisation sector other than up = L/2 mixes two sectors, "
                                     "which the GPU engine does not build");
  if (desc.inversion != 0 && desc.sites > 64)
    raise(QMBED_UNSUPPORTED_BACKEND, "spin inversion sectors are built for chains of at most 64 sites");
  p.inversion = desc.inversion;
  p.symmetric = (p.has_momentum || p.parity != 0 || p.inversion != 0) ? 1 : 0;
  if (p.parity != 0 && p.has_momentum && p.momentum != 0 && 2 * p.momentum != p.sites)
    raise(QMBED_INCOMPATIBLE_SYMMETRY, "parity can share a one-dimensional sector with momentum only at k=0 or k=pi");
  p.n_divisors = 0;
  for (int d = 1; d < p.sites; ++d)
    if (p.sites % d == 0) p.divisors[p.n_divisors++] = d;
  direct_ = !p.symmetric && p.up < 0;
  colex_ = !p.symmetric && p.up >= 0;

  QMBED_CUDA(cudaSetDevice(device_));
  std::vector<uint64_t> binom(static_cast<size_t>(kBinomStride) * kBinomStride, 0);
  for (int n = 0; n < kBinomStride; ++n)
    for (int k = 0; k < kBinomStride; ++k) binom[static_cast<size_t>(n) * kBinomStride + k] = saturating_binomial(n, k);
  binom_.allocate(binom.size() * sizeof(uint64_t));
  QMBED_CUDA(cudaMemcpy(binom_.get(), binom.data(), binom.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));

  // Character table: phase of the physical state T^{-a} rep is
  // exp(-2 pi i k (L - a) / L) (reference coefficient rule, mod.rs:790-806).
  std::vector<double> table(2 * static_cast<size_t>(p.sites));
  for (int a = 0; a < p.sites; ++a) {
    if (!p.has_momentum || p.momentum == 0) {
      table[2 * a] = 1.0;
      table[2 * a + 1] = 0.0;
    } else if (2 * p.momentum == p.sites) {
      table[2 * a] = (a & 1) ? -1.0 : 1.0;  // exact +-1 at k = pi
      table[2 * a + 1] = 0.0;
    } else {
      long long s = (p.sites - a) % p.sites;
      double angle = -(2.0 * M_PI) * static_cast<double>(static_cast<long long>(p.momentum) * s) /
                     static_cast<double>(p.sites);
      table[2 * a] = std::cos(angle);
      table[2 * a + 1] = std::sin(angle);
    }
  }
  phase_.allocate(table.size() * sizeof(double));
  QMBED_CUDA(cudaMemcpy(phase_.get(), table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice));

  if (p.up >= 0) {
    parent_dim_ = saturating_binomial(p.sites, p.up);
    if (parent_dim_ == UINT64_MAX) raise(QMBED_UNSUPPORTED_BACKEND, "sector is too large to enumerate");
  } else {
    if (p.sites > 40) raise(QMBED_UNSUPPORTED_BACKEND, "enumerating the unconstrained Hilbert space is infeasible");
    parent_dim_ = 1ULL << p.sites;
  }
  if (direct_) {
    dim_ = parent_dim_;
  } else if (words() == 1) {
    enumerate<uint64_t>();
  } else {
    enumerate<u128>();
  }
  prepare_lookup();
  QMBED_CUDA(cudaDeviceSynchronize());
  build_seconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

template <typename S>
void SpinBasis::enumerate() {
  const uint64_t total = parent_dim_;
  const uint64_t threads = (total + kEnumChunk - 1) / kEnumChunk;
  const uint64_t blocks = (threads + kEnumThreads - 1) / kEnumThreads;
  if (blocks > 0x7fffffffULL) raise(QMBED_UNSUPPORTED_BACKEND, "sector is too large to enumerate");
  DeviceBuffer counts(threads * sizeof(uint8_t));
  DeviceBuffer totals(blocks * sizeof(uint32_t));
  enumerate_count_kernel<S><<<static_cast<unsigned>(blocks), kEnumThreads>>>(params_, total, binom_.as<uint64_t>(),
                                                                             counts.as<uint8_t>(),
                                                                             totals.as<uint32_t>());
  QMBED_LAUNCH_CHECK();
  std::vector<uint32_t> host_totals(blocks);
  QMBED_CUDA(cudaMemcpy(host_totals.data(), totals.get(), blocks * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  std::vector<uint64_t> offsets(blocks);
  uint64_t running = 0;
  for (uint64_t b = 0; b < blocks; ++b) {
    offsets[b] = running;
    running += host_totals[b];
  }
  dim_ = running;
  DeviceBuffer device_offsets(blocks * sizeof(uint64_t));
  QMBED_CUDA(cudaMemcpy(device_offsets.get(), offsets.data(), blocks * sizeof(uint64_t), cudaMemcpyHostToDevice));
  states_.allocate(std::max<uint64_t>(dim_, 1) * sizeof(S));
  if (params_.symmetric) orbits_.allocate(std::max<uint64_t>(dim_, 1) * sizeof(uint16_t));
  enumerate_fill_kernel<S><<<static_cast<unsigned>(blocks), kEnumThreads>>>(
      params_, total, binom_.as<uint64_t>(), counts.as<uint8_t>(), device_offsets.as<uint64_t>(), states_.as<S>(),
      params_.symmetric ? orbits_.as<uint16_t>() : nullptr);
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaDeviceSynchronize());
}

void SpinBasis::copy_states(uint64_t offset, uint64_t count, uint64_t* lo, uint64_t* hi, uint16_t* orbit) const {
  if (offset > dim_ || count > dim_ - offset) raise(QMBED_DIMENSION_MISMATCH, "state range exceeds the basis");
  QMBED_CUDA(cudaSetDevice(device_));
  if (count == 0) return;
  if (direct_) {
    for (uint64_t i = 0; i < count; ++i) {
      if (lo) lo[i] = offset + i;
      if (hi) hi[i] = 0;
      if (orbit) orbit[i] = 1;
    }
    return;
  }
  if (words() == 1) {
    if (lo) QMBED_CUDA(cudaMemcpy(lo, states_.as<uint64_t>() + offset, count * 8, cudaMemcpyDeviceToHost));
    if (hi)
      for (uint64_t i = 0; i < count; ++i) hi[i] = 0;
  } else {
    std::vector<u128> buffer(count);
    QMBED_CUDA(cudaMemcpy(buffer.data(), states_.as<u128>() + offset, count * 16, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < count; ++i) {
      if (lo) lo[i] = static_cast<uint64_t>(buffer[i]);
      if (hi) hi[i] = static_cast<uint64_t>(buffer[i] >> 64);
    }
  }
  if (orbit) {
    if (params_.symmetric)
      QMBED_CUDA(cudaMemcpy(orbit, orbits_.as<uint16_t>() + offset, count * 2, cudaMemcpyDeviceToHost));
    else
      for (uint64_t i = 0; i < count; ++i) orbit[i] = 1;
  }
}

void SpinBasis::images(const uint64_t* lo, const uint64_t* hi, uint64_t n, int64_t* index, double* phase,
                       uint16_t* orbit) const {
  if (n == 0) return;
  QMBED_CUDA(cudaSetDevice(device_));
  DeviceBuffer d_lo(n * 8), d_hi(n * 8), d_index(n * 8), d_phase(n * 16), d_orbit(n * 2);
  QMBED_CUDA(cudaMemcpy(d_lo.get(), lo, n * 8, cudaMemcpyHostToDevice));
  if (hi) QMBED_CUDA(cudaMemcpy(d_hi.get(), hi, n * 8, cudaMemcpyHostToDevice));
  else QMBED_CUDA(cudaMemset(d_hi.get(), 0, n * 8));
  unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  if (words() == 1)
    images_kernel<uint64_t><<<blocks, 256>>>(params_, states_.as<uint64_t>(), orbits(), dim_, direct_, colex_,
                                             binomials(), phase_table(), d_lo.as<uint64_t>(), d_hi.as<uint64_t>(), n,
                                             d_index.as<int64_t>(), d_phase.as<double>(), d_orbit.as<uint16_t>());
  else
    images_kernel<u128><<<blocks, 256>>>(params_, states_.as<u128>(), orbits(), dim_, direct_, colex_, binomials(),
                                         phase_table(), d_lo.as<uint64_t>(), d_hi.as<uint64_t>(), n,
                                         d_index.as<int64_t>(), d_phase.as<double>(), d_orbit.as<uint16_t>());
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpy(index, d_index.get(), n * 8, cudaMemcpyDeviceToHost));
  QMBED_CUDA(cudaMemcpy(phase, d_phase.get(), n * 16, cudaMemcpyDeviceToHost));
  QMBED_CUDA(cudaMemcpy(orbit, d_orbit.get(), n * 2, cudaMemcpyDeviceToHost));
}

}  // namespace qmbed
