// Spin-chain Hamiltonian on a sector basis: matrix-free action and packed
// sparse storage, both built from the same per-row term expansion.
#pragma once

#include <complex>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "basis.cuh"
#include "flipchain.cuh"
#include "hv_tile.cuh"

namespace qmbed {

using C64 = std::complex<double>;

struct CouplingDesc {
  C64 coefficient;
  std::vector<int> sites;
};

// One local operator product (reference OperatorSpec, src/operator/mod.rs:195-319).
struct TermDesc {
  std::string symbols;  // one character per site: I z + - x y (reference LocalOperator::symbol)
  std::vector<CouplingDesc> couplings;
};

// One coupling of one product, ready for the device. `sym`/`site` are the
// product in application order: position n-1 acts first, like the reference
// visit loop (src/basis/mod.rs:1150-1228).
struct Instance {
  double cr, ci;   // coefficient used in the column-form value
  int n;           // arity
  int diagonal;    // every symbol is I or z: the target is the source state
  char sym[kMaxArity];
  uint8_t site[kMaxArity];
};

struct LocalFactors {
  double z[2];       // z action on digit 0 / 1
  double raise;      // + on digit 0
  double lower;      // - on digit 1
  double xy_scale;   // x/y branch scale
};

enum StorageKind : int {
  kStorageMatrixFree = 0,  // expand terms on every application
  kStoragePacked = 1,      // u32 entries: column | value code << column bits (real operators)
  kStorageWide = 2,        // u32 columns + explicit values
};

enum Precision : int { kFP64 = 64, kFP32 = 32 };

struct OperatorChecks {
  bool hermiticity = true;
  bool particle_conservation = true;
};

class SpinOperator {
 public:
  SpinOperator(std::shared_ptr<SpinBasis> basis, const std::vector<TermDesc>& terms, const OperatorChecks& checks,
               int storage);

  uint64_t dim() const { return basis_->dim(); }
  bool is_real() const { return real_; }
  int storage() const { return storage_; }
  const SpinBasis& basis() const { return *basis_; }
  std::shared_ptr<SpinBasis> basis_ptr() const { return basis_; }
  uint64_t nnz_offdiag() const { return nnz_off_; }
  int value_codes() const { return n_codes_; }
  double assembly_seconds() const { return assembly_seconds_; }

  // y = H x on device vectors. Real operators take real vectors unless
  // `complex_vectors`; complex operators always take interleaved complex.
  // `force_matrix_free` runs the on-the-fly expansion regardless of storage.
  void apply(int precision, bool complex_vectors, const void* x, void* y, cudaStream_t stream,
             bool force_matrix_free = false) const;

  // Rows row0 .. row0 + rows - 1 of y = H x (real vectors, terms expanded on
  // the fly by the tile kernels): x is the full vector, y holds those rows
  // only. The slab form of a row-partitioned operator across devices.
  void apply_rows(int precision, uint64_t row0, uint64_t rows, const void* x, void* y, cudaStream_t stream) const;

  // The same action with the x / sqrt(R) vector of symmetric stored rows
  // written to caller-provided device memory (`scratch`, `scratch_bytes`)
  // instead of a buffer this object allocates. Paths that need no such
  // vector run exactly as apply().
  void apply_with_scratch(int precision, bool complex_vectors, const void* x, void* y, cudaStream_t stream,
                          void* scratch, size_t scratch_bytes) const;

  // Block action in orbit-scaled coordinates z = x / sqrt(R) on row-major
  // n x nb blocks (nb = 8 or 16, precision 64/32):
  //   out = alpha * (S^-1 H S) z + beta * z + gamma * p     (p may be null; out may alias p, not z)
  // Available for real operators with packed rows (supports_block()).
  // The kernel shape (entry split across lanes, entry batch depth) is chosen
  // per (precision, nb, p given) by timing on the first call (autotuner).
  // Real operators with packed rows (autotuned gather kernel) or matrix-free
  // storage (the expansion shared by the block's columns).
  bool supports_block() const;
  void apply_block(int precision, int nb, const void* z, const void* p, void* out, double alpha, double beta,
                   double gamma, cudaStream_t stream) const;
  // Index of the shape the autotuner chose, or -1 before the first call.
  int tuned_block_shape(int precision, int nb, bool with_p) const;

  // Rows stored with explicit values (storage kStorageWide), for kernels that
  // combine several operators on one basis. The values exclude the orbit
  // factors: in coordinates z = x / sqrt(R) the action is
  // (S^-1 H S z)_r = sum_e values[e] z[cols[e]] + diag[r] z[r].
  struct ExplicitRows {
    uint64_t n = 0;
    bool row_ptr64 = false;
    const void* row_ptr = nullptr;
    const uint32_t* cols = nullptr;
    const double* values = nullptr;  // interleaved complex FP64, one per entry
    const double* diag = nullptr;    // FP64: real (n) for real operators, interleaved complex (2n) otherwise
    bool diag_complex = false;
  };
  ExplicitRows explicit_rows() const;

  // The structured flip-chain action, when this operator has that form
  // (full space, matrix-free storage, z products and single x flips).
  const FlipChain* flip_chain() const { return flip_.get(); }

  // Dense Hermitian check of the assembled operator at tolerance 1e-12
  // (OperatorBuilder::build + is_hermitian, src/operator/mod.rs:2212).
  bool check_hermitian() const;

  // Assembled rows on the host (for tests): row pointer, columns, values.
  void export_csr(std::vector<uint64_t>& row_ptr, std::vector<uint32_t>& cols, std::vector<C64>& values) const;
  // apply_sector_shift (src/operator/mod.rs:2305-2351): these terms applied to
  // a vector of this operator's basis (the source) and reduced into `target`
  // (same sites, same device). x: source dimension, y: target dimension,
  // both interleaved complex FP64 on the device; y is overwritten.
  void apply_shift(const SpinBasis& target, const double* x, double* y, cudaStream_t stream) const;

  // Exact stored 1-norm and trace shift (shifted_trace_and_one_norm,
  // src/solve/mod.rs:59-104), computed on the device.
  void trace_and_one_norm(C64* shift, double* one_norm) const;

  // Bytes per application in the operand model D(b_state + s_y) + (D + nnz_off) s_x.
  double operand_bytes(int precision, bool complex_vectors) const;

  // Lookup used by the on-the-fly action (LookupMode): auto (the basis's
  // image table when built, else the representative search), table (built
  // here if absent; raises when it does not fit), search, or legacy (the
  // one-thread-per-row expansion of every product, kept for u128 states and
  // products that repeat a site).
  void set_lookup(int mode);
  int lookup_mode() const { return lookup_mode_; }
  // What the on-the-fly action runs now: 1 table, 2 search, 3 legacy,
  // 4 direct/colex (no symmetry).
  int lookup_in_use() const;
  // True when the on-the-fly action takes the translation-structured (chain)
  // form of its flip program.
  bool chain_form() const { return prog_.ok() && prog_.chain_ok(); }

 private:
  void build_instances(const std::vector<TermDesc>& terms, const OperatorChecks& checks);
  void assemble();
  void ensure_scratch(int precision, bool complex_vectors) const;
  void launch_block_matrix_free(int precision, int nb, const void* z, const void* p, void* out, double alpha,
                                double beta, double gamma, cudaStream_t stream) const;
  void launch_block(int shape, int precision, int nb, const void* z, const void* p, void* out, double alpha,
                    double beta, double gamma, cudaStream_t stream) const;
  int block_shape(int precision, int nb, const void* z, const void* p, double alpha, double beta, double gamma,
                  cudaStream_t stream) const;

  std::shared_ptr<SpinBasis> basis_;
  int storage_;
  bool real_ = true;
  LocalFactors factors_{};
  int n_inst_ = 0;
  DeviceBuffer inst_adj_, inst_fwd_;
  DeviceBuffer inv_sqrt_;   // 257 doubles: 1/sqrt(R)
  // Assembled storage.
  uint64_t nnz_off_ = 0;
  int col_bits_ = 0, n_codes_ = 0;
  bool row_ptr64_ = false;
  DeviceBuffer row_ptr_, entries_, values64_, values32_, code_table_, diag64_, diag32_;
  double assembly_seconds_ = 0.0;
  mutable DeviceBuffer scaled_x_;   // x / sqrt(R) for symmetric packed storage
  mutable size_t scaled_bytes_ = 0;
  std::unique_ptr<FlipChain> flip_;
  mutable std::mutex tune_mu_;
  mutable std::map<int, int> block_shapes_;  // autotuned block-action shape per key
  DeviceFlipProgram prog_;                   // flip form of the adjoint products (u64 states)
  int lookup_mode_ = kLookupAuto;
  // The warp-tile kernel with the current lookup; false when it does not apply.
  bool launch_tile_action(const TileLaunch& l) const;
  // Off-diagonal nonzeros after coalescing of a matrix-free operator, counted
  // on the device on first use.
  uint64_t count_offdiag() const;
  mutable uint64_t counted_nnz_ = ~0ull;
};

}  // namespace qmbed
