// Structured action of full-space spin-1/2 chains whose terms are products of
// z (diagonal) or a single x (one bit flip): transverse-field Ising chains and
// their relatives. No matrix is stored: the diagonal is evaluated from the bits
// of the state index, and one pass over shared-memory tiles of consecutive
// elements serves the low-bit flips from the tile and the high-bit flips from
// coalesced reads of the partner tiles.
#pragma once

#include <complex>
#include <memory>
#include <vector>

#include "common.cuh"

namespace qmbed {

struct FlipChainDesc {
  int sites = 0;
  std::vector<uint64_t> z_masks;   // diagonal products: sites of the z factors
  std::vector<double> z_coefs;     // coefficient x z1^|mask|, so D(s) = sum c (-1)^popcount(~s & mask)
  std::vector<double> x_coefs;     // per site: amplitude of the single flip of that bit
};

// out = alpha * (H x) + beta * x + gamma * p + kappa * q  on full-space
// vectors (real or interleaved complex, FP64 or FP32); p and q may be null;
// out may alias p (rows are read before they are written), never x or q.
// kappa is complex (applied to complex vectors; its real part for real ones).
struct FlipStep {
  double alpha = 1.0, beta = 0.0, gamma = 0.0;
  double kappa_re = 0.0, kappa_im = 0.0;
};

// Runs the multi-pass action's bounded stage wait on a barrier that no copy
// completes (1024 polls) on `device`; returns 1 when it gave up as designed.
int flip_stage_wait_selftest(int device);

class FlipChain {
 public:
  explicit FlipChain(const FlipChainDesc& d);
  uint64_t dim() const { return 1ull << sites_; }
  int sites() const { return sites_; }
  // y = H x (step = identity coefficients) or the fused three/four-term form.
  void apply(int precision, bool cplx, const void* x, void* out, const void* p, const void* q, const FlipStep& step,
             cudaStream_t stream) const;
  // Gershgorin-type bounds: |D| max over the diagonal terms plus sum |x|.
  double norm_bound() const;
  // Raises when a multi-pass launch recorded a timed-out tile wait (and clears it).
  void check_status() const;

 private:
  int sites_;
  int n_diag_;
  DeviceBuffer diag_masks_, diag_coefs_, x_coefs_;
  mutable DeviceBuffer tables_;  // low-bit diagonal tables (FP64, FP32)
  mutable size_t tables_bytes_ = 0;
  mutable int tables_ready_ = 0;  // bit 1: FP64 table, bit 2: FP32 table
  mutable int table_tb_[2] = {0, 0};
  // multi-pass action (vectors beyond the L2): low-bit tables of its box width, time-out status
  void apply_multipass(int precision, bool cplx, const void* x, void* out, const void* p, const void* q,
                       const FlipStep& step, cudaStream_t stream, int sms) const;
  mutable DeviceBuffer pass_tables_[2], pass_high_tables_[2];
  mutable size_t pass_table_bytes_[2] = {0, 0};
  mutable int pass_table_tb_[2] = {0, 0};
  DeviceBuffer status_;
  std::vector<double> host_diag_coefs_, host_x_;
};

}  // namespace qmbed
