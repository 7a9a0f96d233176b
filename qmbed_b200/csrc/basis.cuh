// Spin-1/2 chain sector basis resident in HBM.
#pragma once

#include <memory>
#include <mutex>

#include "common.cuh"

namespace qmbed {

enum Normalization : int { kAngularMomentum = 0, kPauli = 1, kPauliCartesian = 2 };

struct SpinBasisDesc {
  int sites;
  int up;            // -1: no fixed magnetisation
  int has_momentum;
  int momentum;      // any integer; canonicalised modulo L
  int parity;        // 0 none, +-1
  int normalization; // Normalization
  int inversion;     // 0 none, +-1: global spin-flip sector (up = L/2 or the full space, L <= 64)
};

// Image table of a symmetry sector: one entry per state of the parent space
// (indexed by colex rank for fixed weight, by the state itself otherwise):
//   entry = row | code << idx_bits,  code = sign | orbit class << 1 | m << (1 + rbits)
// where row is the representative's index, sign and m give the character of
// the group element mapping the state to its representative (m indexes
// exp(-2 pi i m / L); m is absent for real characters) and the orbit class
// indexes the sector's possible orbit sizes. States outside the sector hold
// all ones. u32 entries when the fields fit 32 bits, u64 otherwise.
struct ImageTable {
  DeviceBuffer entries;
  uint64_t length = 0, bytes = 0;
  bool wide = false;
  int idx_bits = 0, rbits = 0, mbits = 0;
  DeviceBuffer class_inv_sqrt;  // per orbit class: 1/sqrt(R)
  DeviceBuffer class_sizes;     // per orbit class: R (u16)
  DeviceBuffer phase_m;         // 2L doubles
  double build_seconds = 0.0;
};

// Layout in HBM:
//   states : dim x u64 (L <= 64) or dim x u128 (L <= 128), ascending. Absent
//            for the full space without symmetry, where state == index.
//   orbits : dim x u16 orbit sizes R (absent when every R is 1).
//   binom  : (L+1) x (L+1) u64 binomials, saturated, for colex rank/unrank.
class SpinBasis {
 public:
  explicit SpinBasis(const SpinBasisDesc& desc, int device);
  ~SpinBasis() = default;

  int device() const { return device_; }
  int sites() const { return params_.sites; }
  int words() const { return params_.sites <= 64 ? 1 : 2; }
  uint64_t dim() const { return dim_; }
  const SectorParams& params() const { return params_; }
  int normalization() const { return normalization_; }
  bool direct() const { return direct_; }   // state == index
  bool colex() const { return colex_; }     // index = colex rank
  bool symmetric() const { return params_.symmetric != 0; }
  const void* states() const { return states_.get(); }
  const uint16_t* orbits() const { return orbits_.as<uint16_t>(); }
  const uint64_t* binomials() const { return binom_.as<uint64_t>(); }
  const double* phase_table() const { return phase_.as<double>(); }  // 2L doubles: exp(2 pi i k a / L)
  bool real_phases() const { return !params_.has_momentum || params_.momentum == 0 || 2 * params_.momentum == params_.sites; }

  // Copies [offset, offset+count) states (as lo/hi u64 words) and orbit
  // sizes to host arrays (either pointer may be null).
  void copy_states(uint64_t offset, uint64_t count, uint64_t* lo, uint64_t* hi, uint16_t* orbit) const;
  // Maps physical states to (row index or -1, phase, orbit size) on the GPU.
  void images(const uint64_t* lo, const uint64_t* hi, uint64_t n, int64_t* index, double* phase,
              uint16_t* orbit) const;
  double build_seconds() const { return build_seconds_; }
  uint64_t parent_dim() const { return parent_dim_; }

  // Lookup structures of the warp-tile H.v (u64 states only). Colex chunk
  // tables of fixed-weight spaces (4-bit chunks, stride up + 1; absent when
  // larger than 40 KB) and fence keys (every fence_segment()-th
  // representative, at most 4096) are built with the basis.
  const uint64_t* rank_chunk_table() const { return rank_tab_.as<uint64_t>(); }
  int rank_chunk_count() const { return rank_chunks_; }
  int rank_chunk_stride() const { return rank_stride_; }
  const uint64_t* fence_keys() const { return fences_.as<uint64_t>(); }
  int fence_count() const { return n_fences_; }
  uint64_t fence_segment() const { return fence_seg_; }
  int fence_levels() const { return fence_levels_; }
  // The image table when built, else null. build_image_table builds it once
  // (thread-safe) when it fits QMBED_IMAGE_TABLE_MAX_BYTES (default 48 GiB)
  // and 60% of the free device memory; otherwise it returns null, or raises
  // when `required`.
  const ImageTable* image_table() const;
  const ImageTable* build_image_table(bool required) const;
  // images() resolved through the image table (built here if absent): u64
  // states of a symmetry sector only.
  void table_images(const uint64_t* lo, uint64_t n, int64_t* index, double* phase, uint16_t* orbit) const;

 private:
  template <typename S>
  void enumerate();
  void prepare_lookup();

  int device_;
  SectorParams params_{};
  int normalization_;
  bool direct_ = false, colex_ = false;
  uint64_t dim_ = 0, parent_dim_ = 0;
  DeviceBuffer states_, orbits_, binom_, phase_;
  double build_seconds_ = 0.0;
  DeviceBuffer rank_tab_, fences_;
  int rank_chunks_ = 0, rank_stride_ = 0, n_fences_ = 0, fence_levels_ = 0;
  uint64_t fence_seg_ = 0;
  mutable std::mutex table_mu_;
  mutable std::unique_ptr<ImageTable> table_;
};

}  // namespace qmbed
