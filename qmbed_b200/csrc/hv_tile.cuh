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

enum GroupKind : uint8_t { kGroupGeneric = 0, kGroupPair = 1 };

// Products sharing one flip mask. A pair group's amplitude depends on the
// digits of two sites only (i <= j, i == j for one site), so it is a 4-entry
// table indexed by d_i | d_j << 1; generic groups keep their terms.
struct FlipGroup {
  uint64_t flip;
  uint32_t first;      // generic: first term; pair: amplitude slot
  uint16_t count;      // generic: term count
  uint8_t kind;        // GroupKind
  uint8_t nz;          // pair: bit v set when the amplitude at digits v is nonzero
  uint8_t site_i, site_j;
  uint8_t chunk_lo, chunk_hi;  // 4-bit chunks holding the lowest / highest flipped bit
  uint8_t pad[4];
};
static_assert(sizeof(FlipGroup) == 24, "FlipGroup is packed for shared memory");

// Translation-structured form of a program whose products all act on bonds
// (i, i + d mod L) with the same amplitude table for every bond of one
// displacement d (uniform chains: Heisenberg, XXZ, J1-J2, XY, DM, ...).
// For a class, B = state rotated so that bit i of B is digit i + d; the
// digits of every bond at once are (bit i of s, bit i of B), so activity
// masks and diagonal sums take a few word operations per class.
constexpr int kChainMaxOff = 4;
constexpr int kChainMaxDiag = 6;
struct ChainClass {
  uint64_t bonds;  // bit i: bond (i, i + d mod L) present
  int d;
  int nz;          // off-diagonal: digit patterns v = d_i | d_{i+d} << 1 with nonzero amplitude
  double re[4], im[4];
};
struct ChainProgram {
  int n_off = 0, n_diag = 0, has_field = 0, pad = 0;
  uint64_t field_mask = 0;          // single-site diagonal terms, the same on every site listed
  double field_re[2] = {0, 0}, field_im[2] = {0, 0};
  ChainClass off[kChainMaxOff];
  ChainClass diag[kChainMaxDiag];
};

// Host-side compiled program; `ok` is false when some product repeats a site
// (the generic per-instance expansion serves those operators).
struct FlipProgram {
  bool ok = false;
  bool complex_coefs = false;
  std::vector<FlipTerm> diag_terms;   // diagonal products reading three or more sites
  std::vector<uint32_t> diag_pairs;   // site_i | site_j << 8; amplitude slot = position
  std::vector<FlipGroup> groups;      // off-diagonal, ascending flip mask
  std::vector<FlipTerm> terms;        // terms of the generic groups
  std::vector<double> amp_re, amp_im; // 4 per slot: diagonal pairs first, then pair groups
  bool chain_ok = false;
  ChainProgram chain;
};

// `fixed_weight`: the basis holds states of one weight, so flips that change
// the weight are dropped from the activity masks.
FlipProgram compile_flip_program(const std::vector<Instance>& adjoint, const LocalFactors& f, int sites,
                                 bool fixed_weight);

// kLookupTableGeneric: the image table with the general tile kernel even
// where the nearest-neighbour hop kernel applies (kept for comparisons).
enum LookupMode : int { kLookupAuto = 0, kLookupTable = 1, kLookupSearch = 2, kLookupLegacy = 3,
                        kLookupTableGeneric = 4 };


// Device copy of a flip program, one buffer the kernel stages in shared
// memory: [generic terms][groups][amp_re][amp_im][diagonal pair sites].
class DeviceFlipProgram {
 public:
  void upload(const FlipProgram& prog);
  bool ok() const { return ok_; }
  bool complex_coefs() const { return complex_; }
  const void* data() const { return buf_.get(); }
  size_t bytes() const { return bytes_; }
  int n_dterms() const { return n_dterms_; }
  int n_terms() const { return n_terms_; }
  int n_groups() const { return n_groups_; }
  int n_slots() const { return n_slots_; }
  int n_dpairs() const { return n_dpairs_; }
  size_t groups_offset() const { return groups_offset_; }
  size_t amp_offset() const { return amp_offset_; }
  size_t pairs_offset() const { return pairs_offset_; }
  bool chain_ok() const { return chain_ok_; }
  const ChainProgram& chain() const { return chain_; }

 private:
  bool ok_ = false, complex_ = false, chain_ok_ = false;
  ChainProgram chain_;
  int n_dterms_ = 0, n_terms_ = 0, n_groups_ = 0, n_slots_ = 0, n_dpairs_ = 0;
  size_t groups_offset_ = 0, amp_offset_ = 0, pairs_offset_ = 0, bytes_ = 0;
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
  // Rows computed: row0 .. row0 + rows - 1 (clipped to the dimension). x (or
  // z) is the full vector; y, p and the output block hold these rows only.
  uint64_t row0 = 0, rows = ~0ull;
};

// Runs the tile kernel with the lookup `mode` (auto: the table when the
// basis holds one, else search). Returns false when the operator or basis is
// outside the kernel's scope (u128 states, no flip program, requested table
// absent), in which case nothing was launched.
bool launch_tile(const SpinBasis& basis, const DeviceFlipProgram& prog, int mode, const TileLaunch& a);

// True when the nearest-neighbour hop kernel serves this operator on this
// basis: a chain program whose only off-diagonal class is the bond (i, i + 1),
// a real fixed-weight sector and a 32-bit image table without phase index.
bool hop_kernel_applies(const SpinBasis& basis, const DeviceFlipProgram& prog);

// True when this basis can hold an image table within `limit_bytes`.
bool image_table_feasible(const SpinBasis& basis, uint64_t limit_bytes, uint64_t* bytes_out);

}  // namespace qmbed
