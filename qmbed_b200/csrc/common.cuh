// Shared definitions for the B200 spin-chain engine: error plumbing, device
// buffers, and the bit-level state operations used by every kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace qmbed {

// Error categories mirror the reference `QmbedError` (src/error.rs:4-35); the
// numeric codes are this library's C-ABI status values.
enum Status : int {
  QMBED_OK = 0,
  QMBED_INVALID_OPERATOR = 1,
  QMBED_INVALID_COUPLING = 2,
  QMBED_INVALID_SITE = 3,
  QMBED_STATE_NOT_IN_BASIS = 4,
  QMBED_INVALID_SECTOR = 5,
  QMBED_INCOMPATIBLE_SYMMETRY = 6,
  QMBED_NON_HERMITIAN = 7,
  QMBED_INVALID_OPTIONS = 8,
  QMBED_DIMENSION_MISMATCH = 9,
  QMBED_RANK_DEFICIENT = 10,
  QMBED_UNSUPPORTED_BACKEND = 11,
  QMBED_INTERNAL_STATE = 13,
  QMBED_NON_CONVERGENCE = 14,
  QMBED_CUDA_ERROR = 20,
  QMBED_DEVICE_TIMEOUT = 21,
};

struct Error : std::runtime_error {
  int code;
  size_t iterations = 0;
  double residual = 0.0;
  Error(int c, const std::string& message) : std::runtime_error(message), code(c) {}
};

// Builds the Display text of the matching reference error variant.
[[noreturn]] void raise(int code, const std::string& detail);
[[noreturn]] void raise_nonconvergence(size_t iterations, double residual);

#define QMBED_CUDA(call)                                                                     \
  do {                                                                                       \
    cudaError_t qmbed_status_ = (call);                                                      \
    if (qmbed_status_ != cudaSuccess)                                                        \
      ::qmbed::raise(::qmbed::QMBED_CUDA_ERROR,                                              \
                     std::string(#call) + ": " + cudaGetErrorString(qmbed_status_));         \
  } while (0)

// Every kernel launch in the library is followed by exactly one
// QMBED_LAUNCH_CHECK, which also counts it (qmbed_gpu_launch_count).
void count_launch();
#define QMBED_LAUNCH_CHECK()          \
  do {                                \
    ::qmbed::count_launch();          \
    QMBED_CUDA(cudaGetLastError());   \
  } while (0)

// Owning device allocation. The engine allocates once per basis/operator/solve
// and reuses buffers across iterations.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { allocate(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& other) noexcept : ptr_(other.ptr_), bytes_(other.bytes_) {
    other.ptr_ = nullptr;
    other.bytes_ = 0;
  }
  DeviceBuffer& operator=(DeviceBuffer&& other) noexcept {
    if (this != &other) {
      release();
      ptr_ = other.ptr_;
      bytes_ = other.bytes_;
      other.ptr_ = nullptr;
      other.bytes_ = 0;
    }
    return *this;
  }
  void allocate(size_t bytes);
  void release();
  template <typename T>
  T* as() const { return static_cast<T*>(ptr_); }
  void* get() const { return ptr_; }
  size_t bytes() const { return bytes_; }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

constexpr int kMaxArity = 8;
constexpr int kMaxSites = 128;

// ---------------------------------------------------------------------------
// Bit-level state operations (u64 for L <= 64, u128 for L <= 128).
// ---------------------------------------------------------------------------
using u128 = unsigned __int128;

template <typename S>
__host__ __device__ inline S low_mask(int sites) {
  return sites >= static_cast<int>(8 * sizeof(S)) ? ~static_cast<S>(0) : ((static_cast<S>(1) << sites) - 1);
}

// Translation by `shift` sites: site i -> i + shift (mod L), the base-2 fast
// path of rotate_lattice_state (reference src/basis/mod.rs:661-686).
template <typename S>
__host__ __device__ inline S rotate_state(S state, int shift, int sites, S mask) {
  if (shift == 0) return state;
  return ((state << shift) & mask) | (state >> (sites - shift));
}

__host__ __device__ inline uint64_t bit_reverse64(uint64_t v) {
#ifdef __CUDA_ARCH__
  return __brevll(v);
#else
  v = ((v >> 1) & 0x5555555555555555ULL) | ((v & 0x5555555555555555ULL) << 1);
  v = ((v >> 2) & 0x3333333333333333ULL) | ((v & 0x3333333333333333ULL) << 2);
  v = ((v >> 4) & 0x0F0F0F0F0F0F0F0FULL) | ((v & 0x0F0F0F0F0F0F0F0FULL) << 4);
  v = ((v >> 8) & 0x00FF00FF00FF00FFULL) | ((v & 0x00FF00FF00FF00FFULL) << 8);
  v = ((v >> 16) & 0x0000FFFF0000FFFFULL) | ((v & 0x0000FFFF0000FFFFULL) << 16);
  return (v >> 32) | (v << 32);
#endif
}

// Reflection site -> L-1-site (reference reflect_lattice_state, 688-698).
__host__ __device__ inline uint64_t reflect_state(uint64_t state, int sites) {
  return bit_reverse64(state) >> (64 - sites);
}
__host__ __device__ inline u128 reflect_state(u128 state, int sites) {
  uint64_t lo = static_cast<uint64_t>(state), hi = static_cast<uint64_t>(state >> 64);
  u128 r = (static_cast<u128>(bit_reverse64(lo)) << 64) | bit_reverse64(hi);
  return r >> (128 - sites);
}

__host__ __device__ inline int popcount_state(uint64_t v) {
#ifdef __CUDA_ARCH__
  return __popcll(v);
#else
  return __builtin_popcountll(v);
#endif
}
__host__ __device__ inline int popcount_state(u128 v) {
  return popcount_state(static_cast<uint64_t>(v)) + popcount_state(static_cast<uint64_t>(v >> 64));
}

// ---------------------------------------------------------------------------
// Sector description shared by basis enumeration and operator kernels.
// ---------------------------------------------------------------------------
struct SectorParams {
  int sites;
  int up;             // fixed number of up spins, -1 for none
  int has_momentum;   // translation sector selected
  int momentum;       // canonical k in [0, L)
  int parity;         // 0 none, else +-1
  int inversion;      // 0 none, else +-1: character of the global spin flip (every bit inverted)
  int symmetric;      // has_momentum || parity || inversion
  int n_divisors;     // proper divisors of L in increasing order (periods)
  int divisors[32];
};

// Result of mapping a physical state onto its sector representative.
template <typename S>
struct Canonical {
  S rep;          // minimum of the orbit (reference rep = min, mod.rs:785-788)
  int shift;      // rotate(t' or reflect(t'), shift) == rep, t' = t or its spin flip
  int reflected;  // 1 if the minimum came from the reflected state
  int inverted;   // 1 if the minimum came from the spin-flipped state
};

// Folds the translations (and reflections) of `t` into `best`, starting at
// shift `first_shift`.
template <typename S>
__host__ __device__ inline void scan_orbit(S t, const SectorParams& p, S mask, int first_shift, int inverted,
                                           Canonical<S>& best) {
  const int translations = p.has_momentum ? p.sites : 1;
  for (int s = first_shift; s < translations; ++s) {
    S r = rotate_state(t, s, p.sites, mask);
    if (r < best.rep) best = Canonical<S>{r, s, 0, inverted};
  }
  if (p.parity != 0) {
    S u = reflect_state(t, p.sites);
    for (int s = 0; s < translations; ++s) {
      S r = rotate_state(u, s, p.sites, mask);
      if (r < best.rep) best = Canonical<S>{r, s, 1, inverted};
    }
  }
}

// Minimum over translations (and reflections, and the global spin flip) of
// `t`, with the group element that reaches it. Translation-only sectors use
// shifts 0..L-1; parity-only sectors use {t, reflect(t)}; the spin flip
// doubles the scan with ~t (it commutes with every site permutation).
template <typename S>
__host__ __device__ inline Canonical<S> canonicalize(S t, const SectorParams& p, S mask) {
  Canonical<S> best{t, 0, 0, 0};
  scan_orbit(t, p, mask, 1, 0, best);
  if (p.inversion != 0) scan_orbit(static_cast<S>(~t & mask), p, mask, 0, 1, best);
  return best;
}

// Smallest period of a state under translation (a divisor of L).
template <typename S>
__host__ __device__ inline int translation_period(S rep, const SectorParams& p, S mask) {
  if (!p.has_momentum) return 1;
  for (int i = 0; i < p.n_divisors; ++i) {
    int d = p.divisors[i];
    if (rotate_state(rep, d, p.sites, mask) == rep) return d;
  }
  return p.sites;
}

// Orbit size R and sector compatibility of a representative, following the
// one-dimensional projection rules of spin_symmetry_sector (mod.rs:785-841):
// an orbit belongs to the sector iff its projected coefficients are nonzero.
template <typename S>
__host__ __device__ inline int lattice_orbit_size_if_compatible(S rep, const SectorParams& p, S mask) {
  int period = translation_period(rep, p, mask);
  if (p.has_momentum && (static_cast<long long>(p.momentum) * period) % p.sites != 0) return 0;
  if (p.parity == 0) return period;
  S u = reflect_state(rep, p.sites);
  const int translations = p.has_momentum ? p.sites : 1;
  int self_shift = -1;
  for (int s = 0; s < translations && s < period; ++s) {
    if (rotate_state(u, s, p.sites, mask) == rep) { self_shift = s; break; }
  }
  if (self_shift < 0) return 2 * period;  // reflection gives a distinct orbit
  // reflect(rep) = T^{-b} rep: the coefficient is chi(s)(1 + p chi(b)), with
  // chi(b) = exp(2 pi i k b / L) real (+-1) because k is 0 or L/2 here.
  int sign = 1;
  if (p.has_momentum && 2 * p.momentum == p.sites && (self_shift & 1)) sign = -1;
  return (p.parity * sign == 1) ? period : 0;
}

// Character exp(-2 pi i k s / L) of T^s when it is real (+-1); 2 otherwise.
__host__ __device__ inline int real_translation_character(int s, const SectorParams& p) {
  if (!p.has_momentum) return 1;
  const long long m = (static_cast<long long>(p.momentum) * s) % p.sites;
  if (m == 0) return 1;
  return 2 * m == p.sites ? -1 : 2;
}

// Orbit size and compatibility with the spin flip Z (character z) added to
// the lattice group G: if Z rep = g rep for some g in G, the stabiliser holds
// g^-1 Z and the orbit belongs to the sector iff chi(g) = z (then its size is
// that of the G orbit); otherwise Z doubles the orbit. This is the
// one-dimensional orbit rule of the reference's general reducer
// (trace_symmetry_orbit, src/basis/mod.rs:3455-3538) for these generators.
template <typename S>
__host__ __device__ inline int orbit_size_if_compatible(S rep, const SectorParams& p, S mask) {
  const int base = lattice_orbit_size_if_compatible(rep, p, mask);
  if (base == 0 || p.inversion == 0) return base;
  const S flipped = static_cast<S>(~rep & mask);
  const int translations = p.has_momentum ? p.sites : 1;
  int character = 0;
  for (int s = 0; s < translations && character == 0; ++s)
    if (rotate_state(rep, s, p.sites, mask) == flipped) character = real_translation_character(s, p);
  if (character == 0 && p.parity != 0) {
    const S u = reflect_state(rep, p.sites);
    for (int s = 0; s < translations && character == 0; ++s)
      if (rotate_state(u, s, p.sites, mask) == flipped) {
        character = real_translation_character(s, p);
        if (character != 2) character *= p.parity;
      }
  }
  if (character == 0) return 2 * base;
  return character == p.inversion ? base : 0;
}

}  // namespace qmbed
