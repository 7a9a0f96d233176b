// Matrix-free H.v on u64 states, one warp per tile of 32 consecutive rows.
//
// The operator's adjoint products are compiled once into a flip program:
// each product of spin-1/2 factors on distinct sites acts on a basis state s
// as  s -> s ^ flip  with amplitude  k * (-1)^popcount(~s & sign_mask)  when
// (s & req_mask) == req_val, and zero otherwise. Products with the same flip
// mask form one group, so a row expands into at most one target per group.
// The lanes of a warp pop their rows' active groups in lockstep and resolve
// each target to (column, character, orbit size) through one of four lookups:
//
//   direct : full space without symmetry, column = state
//   colex  : fixed weight without symmetry, column = colex rank
//   table  : symmetry sector with an image table: one read of
//            table[colex rank of the target] gives column, character and
//            orbit class, with no representative search at all
//   search : symmetry sector without a table: orbit minimum over the group,
//            then a search of the sorted representatives whose first levels
//            come from fence keys staged in shared memory
//
// Reference behaviour: visit_unreduced_local_transitions_with_symbols
// (src/basis/mod.rs:1122-1232), index_transition (1561-1580), apply_real /
// apply (src/operator/mod.rs:1414-1548).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "basis.cuh"

namespace qmbed {

struct Instance;
struct LocalFactors;

// One product in flip form; (kr, ki) = conj(adjoint coefficient x constant
// amplitude), so the H-row entry of target s ^ flip is (kr + i ki) * sign.
struct FlipTerm {
  uint64_t req_mask, req_val, sign_mask;
  double kr, ki;
};

struct FlipGroup {
  uint64_t flip;
  uint32_t first, count;  // terms[first, first + count)
};

// Host-side compiled program; `ok` is false when some product repeats a site
// (the generic per-instance expansion serves those operators).
struct FlipProgram {
  bool ok = false;
  bool complex_coefs = false;
  std::vector<FlipTerm> diag;      // flip == 0
  std::vector<FlipGroup> groups;   // off-diagonal, ascending flip mask
  std::vector<FlipTerm> terms;     // terms of the groups
};

FlipProgram compile_flip_program(const std::vector<Instance>& adjoint, const LocalFactors& f, int sites);

enum LookupMode : int { kLookupAuto = 0, kLookupTable = 1, kLookupSearch = 2, kLookupLegacy = 3 };

// Device copy of a flip program: [diag terms][group terms] then the groups.
class DeviceFlipProgram {
 public:
  void upload(const FlipProgram& prog);
  bool ok() const { return ok_; }
  bool complex_coefs() const { return complex_; }
  const FlipTerm* terms() const { return buf_.as<FlipTerm>(); }
  const FlipGroup* groups() const { return reinterpret_cast<const FlipGroup*>(buf_.as<char>() + groups_offset_); }
  int n_diag() const { return n_diag_; }
  int n_terms() const { return n_terms_; }
  int n_groups() const { return n_groups_; }
  size_t bytes() const { return bytes_; }

 private:
  bool ok_ = false, complex_ = false;
  int n_diag_ = 0, n_terms_ = 0, n_groups_ = 0;
  size_t groups_offset_ = 0, bytes_ = 0;
  DeviceBuffer buf_;
};

// Launch of the tile kernel. NB = 1: y = H x (real or interleaved complex
// vectors, orbit ratios applied). NB = 8 or 16: the block action in
// orbit-scaled coordinates, out = alpha (S^-1 H S z) + beta z + gamma p.
struct TileLaunch {
  int precision = 64;       // 64 or 32
  int nb = 1;
  bool complex_vectors = false;
  const void* x = nullptr;  // x (NB = 1) or z (block)
  const void* p = nullptr;
  void* y = nullptr;
  double alpha = 1.0, beta = 0.0, gamma = 0.0;
  const double* inv_sqrt = nullptr;  // [R] 1/sqrt(R), [257 + R] sqrt(R), R <= 256
  cudaStream_t stream = nullptr;
};

// Runs the tile kernel with the lookup `mode` (auto: the table when the
// basis holds one, else search). Returns false when the operator or basis is
// outside the kernel's scope (u128 states, no flip program, requested table
// absent), in which case nothing was launched.
bool launch_tile(const SpinBasis& basis, const DeviceFlipProgram& prog, int mode, const TileLaunch& a);

// True when this basis can hold an image table within `limit_bytes`.
bool image_table_feasible(const SpinBasis& basis, uint64_t limit_bytes, uint64_t* bytes_out);

}  // namespace qmbed
