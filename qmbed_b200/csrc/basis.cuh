// Spin-1/2 chain sector basis resident in HBM.
#pragma once

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

 private:
  template <typename S>
  void enumerate();

  int device_;
  SectorParams params_{};
  int normalization_;
  bool direct_ = false, colex_ = false;
  uint64_t dim_ = 0, parent_dim_ = 0;
  DeviceBuffer states_, orbits_, binom_, phase_;
  double build_seconds_ = 0.0;
};

}  // namespace qmbed
