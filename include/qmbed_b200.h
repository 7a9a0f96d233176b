/*
 * qmbed_b200 — B200 (sm_100a) engine for QMBED's symmetry-reduced spin-chain
 * Hamiltonian action and the Krylov solvers on it.
 *
 * Two C-ABI surfaces, both exported by libqmbed_b200.so:
 *
 *  1. The drop-in JSON boundary: the same six symbols the reference cdylib
 *     `qmbed-capi` exports (bindings/capi/src/lib.rs:6089-6296) and that the
 *     reference Python package binds at load time
 *     (bindings/python/src/qmbed/_ffi.py:154-186). Requests and responses use
 *     the reference JSON schema; a response string is owned by the caller
 *     and released exactly once with qmbed_string_free.
 *
 *  2. A typed API (qmbed_gpu_*) over opaque handles with plain pointers and
 *     sizes, used by the test suite and the benchmark. Every function returns
 *     0 on success or a status code below; qmbed_gpu_last_error() returns the
 *     message of the last failure on the calling thread.
 *
 * Complex arrays are interleaved (re, im) doubles. Basis states are split in
 * low/high 64-bit words (hi may be NULL for chains of at most 64 sites).
 */
#ifndef QMBED_B200_H
#define QMBED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMBED_API __attribute__((visibility("default")))

/* Status codes: the categories of the reference QmbedError (src/error.rs:4-35). */
enum {
  QMBED_STATUS_OK = 0,
  QMBED_STATUS_INVALID_OPERATOR = 1,
  QMBED_STATUS_INVALID_COUPLING = 2,
  QMBED_STATUS_INVALID_SITE = 3,
  QMBED_STATUS_STATE_NOT_IN_BASIS = 4,
  QMBED_STATUS_INVALID_SECTOR = 5,
  QMBED_STATUS_INCOMPATIBLE_SYMMETRY = 6,
  QMBED_STATUS_NON_HERMITIAN = 7,
  QMBED_STATUS_INVALID_OPTIONS = 8,
  QMBED_STATUS_DIMENSION_MISMATCH = 9,
  QMBED_STATUS_RANK_DEFICIENT = 10,
  QMBED_STATUS_UNSUPPORTED_BACKEND = 11,
  QMBED_STATUS_INTERNAL_STATE = 13,
  QMBED_STATUS_NON_CONVERGENCE = 14,
  QMBED_STATUS_CUDA_ERROR = 20
};

/* Spin normalisation (reference SpinNormalization, src/basis/mod.rs:1006-1014). */
enum { QMBED_ANGULAR_MOMENTUM = 0, QMBED_PAULI = 1, QMBED_PAULI_CARTESIAN = 2 };

/* Operator storage on the device. */
enum {
  QMBED_STORAGE_MATRIX_FREE = 0, /* terms expanded on every application */
  QMBED_STORAGE_PACKED = 1,      /* rows assembled once on the GPU (packed u32 entries when real) */
  QMBED_STORAGE_EXPLICIT = 2     /* rows assembled once with an explicit FP64 value per entry */
};

/* Spectral targets (reference SpectrumTarget, src/solve/mod.rs:332-347). */
enum {
  QMBED_SMALLEST_ALGEBRAIC = 0,
  QMBED_LARGEST_ALGEBRAIC = 1,
  QMBED_SMALLEST_MAGNITUDE = 2,
  QMBED_LARGEST_MAGNITUDE = 3,
  QMBED_BOTH_ENDS = 4,
  QMBED_SHIFT = 5
};

/* Solver modes. */
enum {
  QMBED_MODE_PLAIN_FP64 = 0, /* the reference algorithms in FP64 */
  QMBED_MODE_MIXED = 1,      /* FP32 vectors and H.v, FP64 recurrences, FP64 refinement to tolerance */
  QMBED_MODE_FILTERED = 2    /* block Chebyshev-filtered subspace iteration, FP32 then FP64, for the
                                smallest algebraic pairs of real packed operators; otherwise as MIXED */
};

typedef struct qmbed_basis_s* qmbed_basis;
typedef struct qmbed_operator_s* qmbed_operator;

QMBED_API const char* qmbed_gpu_last_error(void);
QMBED_API int qmbed_gpu_device_count(int* count);
/* Number of kernels this library has launched in the process so far. */
QMBED_API int qmbed_gpu_launch_count(uint64_t* count);

/* SpinBasis1D::builder(sites).up(up).momentum(k).parity(p).build()
 * (reference src/basis/mod.rs:1312-1412, spin one half). up < 0: no fixed
 * magnetisation; parity 0: no reflection sector. */
QMBED_API int qmbed_gpu_spin_basis_create(int device, int sites, int up, int has_momentum, int momentum, int parity,
                                          int normalization, qmbed_basis* out);
QMBED_API int qmbed_gpu_basis_destroy(qmbed_basis basis);
/* Basis::len (src/basis/mod.rs:106). */
QMBED_API int qmbed_gpu_basis_dimension(qmbed_basis basis, uint64_t* dimension);
/* Basis::state over [offset, offset+count) plus the orbit sizes of
 * spin_symmetry_sector (src/basis/mod.rs:715-848); any output may be NULL. */
QMBED_API int qmbed_gpu_basis_states(qmbed_basis basis, uint64_t offset, uint64_t count, uint64_t* lo, uint64_t* hi,
                                     uint16_t* orbit);
/* Basis::reduction_image + Basis::index for physical states
 * (src/basis/mod.rs:1536-1560, 1429-1442): index -1 when the state's orbit is
 * not in the sector; phase is complex (2 doubles per state). */
QMBED_API int qmbed_gpu_basis_images(qmbed_basis basis, const uint64_t* lo, const uint64_t* hi, uint64_t n,
                                     int64_t* index, double* phase, uint16_t* orbit);
QMBED_API int qmbed_gpu_basis_build_seconds(qmbed_basis basis, double* seconds);
/* The same images resolved through the sector's image table (one entry per
 * parent state holding row, character and orbit class), built on first use:
 * the lookup the matrix-free action uses. u64 states of symmetry sectors only
 * (otherwise QMBED_STATUS_UNSUPPORTED_BACKEND). Replaces, like
 * qmbed_gpu_basis_images, the HashMap probe of Basis::reduction_image /
 * index_transition (src/basis/mod.rs:1536-1580), with the table in HBM. */
QMBED_API int qmbed_gpu_basis_table_images(qmbed_basis basis, const uint64_t* lo, uint64_t n, int64_t* index,
                                           double* phase, uint16_t* orbit);

/* OperatorBuilder::on(&basis).terms(...).checks(...).build(format)
 * (src/operator/mod.rs:2040-2216). Terms are flattened: term t has arity[t]
 * symbols (one of "Iz+-xy" each) taken in order from `symbols`, and
 * n_couplings[t] couplings, each with a complex coefficient (2 doubles) and
 * arity[t] site indices taken in order from `sites`. */
QMBED_API int qmbed_gpu_operator_create(qmbed_basis basis, int n_terms, const int* arity, const char* symbols,
                                        const int* n_couplings, const double* coefficients, const int* sites,
                                        int check_hermitian, int check_particles, int storage, qmbed_operator* out);
QMBED_API int qmbed_gpu_operator_destroy(qmbed_operator op);
QMBED_API int qmbed_gpu_operator_info(qmbed_operator op, uint64_t* dimension, int* is_real, int* storage,
                                      uint64_t* nnz_offdiag, int* value_codes, double* assembly_seconds);
/* LinearOperator::apply / apply_real (src/operator/mod.rs:1401-1548) on device
 * buffers of the given precision (64 or 32); complex_vectors selects
 * interleaved complex vectors. stream may be NULL (default stream). */
QMBED_API int qmbed_gpu_operator_apply_device(qmbed_operator op, int precision, int complex_vectors, const void* x,
                                              void* y, void* stream, int force_matrix_free);
/* Rows row0 .. row0 + rows - 1 of y = H x for a matrix-free real operator:
 * x is the full device vector (dimension entries), y receives `rows` entries.
 * The slab of a row-partitioned operator whose x is all-gathered across
 * devices (the reference's distributed profile is rejected,
 * src/runtime.rs:224-228; its GPU slot is RuntimeLinearOperator::apply_on,
 * src/runtime.rs:119-175). */
QMBED_API int qmbed_gpu_operator_apply_rows_device(qmbed_operator op, int precision, uint64_t row0, uint64_t rows,
                                                   const void* x, void* y, void* stream);
/* Block action on row-major n x nb device blocks (nb = 8 or 16), in the
 * orbit-scaled coordinates z = x / sqrt(R) of symmetry sectors (z = x without
 * symmetry): out = alpha * (S^-1 H S) z + beta * z + gamma * p, S = diag(sqrt(R)).
 * p may be NULL; out may equal p but not z. One call is one step of a
 * three-term recurrence over nb vectors (the Chebyshev filter of the
 * QMBED_MODE_FILTERED solver). Real operators with packed or matrix-free
 * storage (otherwise QMBED_STATUS_UNSUPPORTED_BACKEND). No counterpart in the
 * reference, whose operators act on one vector at a time
 * (LinearOperator::apply_real, src/operator/mod.rs:1414-1485). */
QMBED_API int qmbed_gpu_operator_apply_block_device(qmbed_operator op, int precision, int nb, const void* z,
                                                    const void* p, void* out, double alpha, double beta, double gamma,
                                                    void* stream);
/* The same action as qmbed_gpu_operator_apply_device, for callers that cannot
 * let a library allocate device memory (applications that manage all GPU
 * memory through their own pool or budget, or that cannot afford the device
 * synchronisation of cudaMalloc/cudaFree in their loop). No counterpart in the
 * reference: it is an addition of this library. It allocates nothing; the
 * x / sqrt(R) vector of symmetry sectors with stored rows goes to a fixed
 * 32 MiB array in device global memory, reserved on every GPU where the
 * library's device code is loaded and held until the process exits. For those
 * operators vectors are limited to 32 MiB (dimension x (2 if complex) x
 * (8 FP64 | 4 FP32) bytes); larger ones return QMBED_STATUS_DIMENSION_MISMATCH.
 * Other operators (matrix-free storage, no symmetry, flip chains) use no
 * scratch and have no limit; flip chains run the matrix-free tile kernel here,
 * because their structured kernels allocate diagonal tables on first use.
 * The first call on a
 * device looks up the array's device address (once per device, cached); make
 * that first call before any stream capture. All calls share the array and it
 * keeps the last call's contents (each call overwrites the part it reads), so
 * calls that overlap on the GPU (other streams, other host threads) race. */
QMBED_API int qmbed_gpu_operator_apply_device_noalloc(qmbed_operator op, int precision, int complex_vectors,
                                                      const void* x, void* y, void* stream);
/* The same action on host buffers (FP64; complex interleaved when complex_vectors). */
QMBED_API int qmbed_gpu_operator_apply_host(qmbed_operator op, int complex_vectors, const double* x, double* y,
                                            int force_matrix_free);
/* Assembled rows (diagonal included, orbit factors applied) of an operator
 * with stored rows: first call with cols == NULL to get *nnz_total. */
QMBED_API int qmbed_gpu_operator_export_csr(qmbed_operator op, uint64_t* nnz_total, uint64_t* row_ptr, uint32_t* cols,
                                            double* values);
/* Operand-byte model of one application: D(b_state + s_y) + (D + nnz_off) s_x.
 * Matrix-free operators count nnz_off (distinct off-diagonal columns per row)
 * once, on the first call. */
QMBED_API int qmbed_gpu_operator_operand_bytes(qmbed_operator op, int precision, int complex_vectors, double* bytes);
/* Lookup of the matrix-free action (LinearOperator::apply with
 * MatrixFormat::MatrixFree, src/operator/mod.rs:1414-1548, whose index
 * transitions probe a HashMap, src/basis/mod.rs:1561-1580):
 * QMBED_LOOKUP_AUTO (the image table when the basis holds one, else the
 * representative search), QMBED_LOOKUP_TABLE (builds the table; error when it
 * does not fit), QMBED_LOOKUP_SEARCH, QMBED_LOOKUP_LEGACY (one thread per row
 * over every product, the form used for u128 states and products that repeat
 * a site), QMBED_LOOKUP_TABLE_GENERIC (the table with the general tile kernel
 * even where the nearest-neighbour hop kernel applies). */
#define QMBED_LOOKUP_AUTO 0
#define QMBED_LOOKUP_TABLE 1
#define QMBED_LOOKUP_SEARCH 2
#define QMBED_LOOKUP_LEGACY 3
#define QMBED_LOOKUP_TABLE_GENERIC 4
QMBED_API int qmbed_gpu_operator_set_lookup(qmbed_operator op, int mode);
/* What the matrix-free action runs: 1 table, 2 search, 3 legacy, 4 no symmetry
 * (direct or colex index), 5 table with the nearest-neighbour hop kernel; whether it expands the products in their
 * translation-structured form (uniform couplings per bond displacement: one
 * activity mask per displacement from word operations); the basis's image
 * table size and build time (0 when none). */
QMBED_API int qmbed_gpu_operator_lookup_info(qmbed_operator op, int* in_use, int* chain_form, uint64_t* table_bytes,
                                             double* table_seconds);

typedef struct {
  uint64_t eigenpairs;
  int target;
  double shift;
  uint64_t krylov_dimension; /* 0: None */
  double tolerance;
  uint64_t max_iterations;
  uint64_t seed;
  int mode; /* QMBED_MODE_* */
} qmbed_eigsh_options;

typedef struct {
  uint64_t iterations;
  uint64_t reorthogonalization_passes;
  uint64_t conditional_second_passes;
  uint64_t fp32_iterations;
  uint64_t fp64_iterations;
  uint64_t operator_applications;
  int converged;
  int complex_vectors;
} qmbed_eigsh_info;

/* eigsh / eigsh_with_initial_subspace (src/solve/mod.rs:2335-2417). initial
 * holds n_initial host vectors (complex, dimension each) or is NULL;
 * eigenvectors (complex, eigenpairs x dimension) may be NULL. */
QMBED_API int qmbed_gpu_eigsh(qmbed_operator op, const qmbed_eigsh_options* options, const double* initial,
                              int n_initial, double* eigenvalues, double* residuals, double* eigenvectors,
                              qmbed_eigsh_info* info);

/* Spectral hint for eigsh (no reference counterpart: the reference estimates
 * nothing before a solve). lower/upper: an interval believed to hold the
 * spectrum (for example the learned bound network's prediction, padded);
 * gap: the predicted gap above the lowest eigenvalue; restart_keep: Ritz
 * vectors the thick restart keeps per cycle (0: the reference's
 * min(needed, krylov / 2), src/solve/mod.rs:1799); check_steps: Lanczos steps
 * of the check that the filtered mode runs before it trusts the interval (its
 * Ritz values must lie inside it, else the solver's own bound estimate is
 * used). On return, used = 1 when the interval passed the check and set the
 * filter, and bound_applications counts the operator applications spent on
 * spectral bounds. An accepted hint with gap > 0 also places the filter's first
 * cut at lower + nb * gap when that is below the check's Ritz value (nb = 8 or
 * 16, the block width). upper <= lower and restart_keep = 0 give an empty
 * hint: the solve is that of qmbed_gpu_eigsh and the outputs are still set.
 * restart_keep applies to the plain FP64 thick restart (mode
 * QMBED_MODE_FP64); the mixed mode keeps the reference's size in both of its
 * phases. */
typedef struct {
  double lower;
  double upper;
  double gap;
  uint64_t restart_keep;
  int check_steps;
  int used;
  uint64_t bound_applications;
} qmbed_eigsh_hint;

/* qmbed_gpu_eigsh with a spectral hint (no reference counterpart). */
QMBED_API int qmbed_gpu_eigsh_hinted(qmbed_operator op, const qmbed_eigsh_options* options, qmbed_eigsh_hint* hint,
                                     const double* initial, int n_initial, double* eigenvalues, double* residuals,
                                     double* eigenvectors, qmbed_eigsh_info* info);

/* ExpmActionPlan::new (src/solve/mod.rs:126-184): degree, scaling, trace
 * shift (complex) and the exact stored 1-norm of A - shift. */
QMBED_API int qmbed_gpu_expm_plan(qmbed_operator op, double coef_re, double coef_im, uint64_t max_degree,
                                  double tolerance, uint64_t max_substeps, uint64_t* degree, uint64_t* scaling,
                                  double* shift, double* one_norm);
/* ExpmActionPlan::apply (src/solve/mod.rs:198-247) on n_vectors host vectors
 * (complex, dimension each); precision 64 (complex128) or 32 (complex64 working vectors). */
QMBED_API int qmbed_gpu_expm_apply_host(qmbed_operator op, double coef_re, double coef_im, uint64_t max_degree,
                                        double tolerance, uint64_t max_substeps, int precision, const double* input,
                                        double* output, uint64_t n_vectors);

/* evolve / evolve_with_diagnostics with hamiltonian = true (src/solve/mod.rs:
 * 3197-3316, 3374-3406): exp(-i H t) initial at each of n_times nondecreasing
 * times by adaptive Lanczos projections without reorthogonalisation. initial
 * is one host vector (interleaved complex); states receives n_times vectors.
 * diagnostics (may be NULL) receives the 7 EvolutionDiagnostics fields in
 * declaration order (src/solve/mod.rs:2546-2555). */
QMBED_API int qmbed_gpu_evolve(qmbed_operator op, const double* initial, int n_times, const double* times,
                               uint64_t krylov_dimension, double tolerance, uint64_t max_substeps, double* states,
                               double* diagnostics);
/* expm_lanczos (src/solve/mod.rs:3432-3454): exp(-i H time) initial from one
 * Lanczos projection of dimension krylov_dimension; host vectors. */
QMBED_API int qmbed_gpu_expm_lanczos(qmbed_operator op, const double* initial, double time,
                                     uint64_t krylov_dimension, double* out);

/* exp(-i H t) initial at each of n_times nondecreasing times (from 0) by a
 * Chebyshev expansion per interval on the spectral interval [e_min, e_max]
 * (NaN for both: the guaranteed bound +-sum|coefficients|), with working
 * precision 64 (complex128) or 32 (complex64). The same states as evolve /
 * expm_multiply (src/solve/mod.rs:3374-3406, 116-248) within the tolerance;
 * the Chebyshev form has no counterpart in the reference. Operators with the
 * structured flip-chain action only (full space, matrix-free storage, terms
 * that are z products or a single x); otherwise QMBED_STATUS_UNSUPPORTED_BACKEND.
 * states receives every time's state, or only the last one when final_only
 * is nonzero (for long trajectories of large chains). info (may be NULL)
 * receives: H applications, intervals, e_min, e_max used, and the largest
 * drift of the state norm. */
QMBED_API int qmbed_gpu_chebyshev_evolve(qmbed_operator op, const double* initial, int n_times, const double* times,
                                         double e_min, double e_max, double tolerance, int precision, int final_only,
                                         double* states, double* info);
/* The same propagation on a device state: `state` (interleaved complex128,
 * dimension x 2 doubles, device memory) holds the initial state and receives
 * the state at the last time; intermediate times are propagated through but
 * not returned, and nothing crosses to the host. Runs on the operator's
 * stream and returns after it completes. Addition of this library. */
QMBED_API int qmbed_gpu_chebyshev_evolve_device(qmbed_operator op, double* state, int n_times, const double* times,
                                                double e_min, double e_max, double tolerance, int precision,
                                                double* info);

/* Lowest eigenvalues of every H(s, p) = sum_k coefficients[p][k] A_k(s) for
 * n_sectors sectors s and n_points scan points p (<= 64), in one batched
 * Lanczos run: each launch applies every sector's operator to every point.
 * components[s * n_components + k] is A_k of sector s, created with
 * QMBED_STORAGE_EXPLICIT on sector s's basis (all components of a sector share
 * its basis handle). Plain three-term Lanczos in FP64 per pair (no
 * reorthogonalisation; copies of converged Ritz values are merged); a pair is
 * done when its wanted values move less than 1e-3 tolerance max(|E|, 1) in
 * 10 steps, or when its Krylov space is exhausted. eigenvalues receives
 * [sector][point][eigenpairs] (eigenpairs <= 4), steps the Lanczos steps per
 * pair, info (may be NULL) the total steps and the applications summed over
 * pairs. The reference solves each pair with eigsh (src/solve/mod.rs:
 * 2335-2350); the batched form has no counterpart there. */
QMBED_API int qmbed_gpu_scan_lowest(int n_sectors, int n_components, const qmbed_operator* components, int n_points,
                                    const double* coefficients, int eigenpairs, double tolerance, int max_steps,
                                    uint64_t seed, double* eigenvalues, int* steps, double* info);
/* The same scan with its verification outputs: residuals[s][p][i] =
 * ||H v - theta v|| / ||v|| of each reported Ritz pair, computed in FP64 from
 * its Ritz vector (the reference's acceptance test r <= tol max(|theta|, 1),
 * src/solve/mod.rs:1252-1263, holds for every reported pair, otherwise
 * QMBED_STATUS_NON_CONVERGENCE); e_max[s][p] = the largest Ritz value at
 * convergence (an inner estimate of the top of the spectrum); info (11
 * doubles): first-pass steps of the longest pair, first-pass applications,
 * verification applications, CUDA graph used (1/0), first-pass seconds,
 * total seconds, largest relative residual, Ritz copies merged, the
 * autotuned resident blocks per SM of the persistent launch, the fastest
 * tuning chunk's milliseconds (0 when not tuned) and the autotuned rows per
 * warp of its apply phase.
 * residuals and e_max may be NULL. */
QMBED_API int qmbed_gpu_scan_solve(int n_sectors, int n_components, const qmbed_operator* components, int n_points,
                                   const double* coefficients, int eigenpairs, double tolerance, int max_steps,
                                   uint64_t seed, double* eigenvalues, double* residuals, double* e_max, int* steps,
                                   double* info);
/* Test of the persistent scan kernel's grid barrier: launches it with one
 * block fewer than it waits for; *status receives 1 when the bounded spin
 * ended in the time-out status (the kernel returns instead of hanging). */
QMBED_API int qmbed_gpu_scan_barrier_selftest(int device, int* status);
/* Test of the multi-pass flip-chain action's bounded wait on its box copies
 * (no reference counterpart): a barrier armed for bytes that no copy
 * delivers is polled 1024 times; *status receives 1 when the wait gave up
 * (the kernel returns instead of hanging). */
QMBED_API int qmbed_gpu_flip_wait_selftest(int device, int* status);

/* Extreme Ritz values of a steps-step FP64 Lanczos run without
 * reorthogonalisation from deterministic_start(seed) (src/solve/mod.rs:
 * 729-742), as used for spectral bounds: out receives the smallest and largest
 * Ritz values and the residual norms of their Ritz pairs (4 doubles). The
 * Ritz values lie inside the spectrum. No counterpart in the reference, whose
 * Lanczos routines return converged eigenpairs only. */
QMBED_API int qmbed_gpu_lanczos_extremes(qmbed_operator op, int steps, uint64_t seed, double* out);

/* Learned spectral bounds: a fully connected ReLU network (inputs ->
 * hidden_layers x width -> outputs, FP32) trained and evaluated by this
 * library's own GPU kernels. It maps model parameters (size, couplings,
 * statistics of random fields) to spectral bounds that set the Chebyshev
 * interval and degree; every prediction used by a solver is checked by a short
 * Lanczos run first. No counterpart in the reference. Parameters are
 * flattened per linear map: W (in x out, row-major) then b (out). */
typedef struct qmbed_mlp_s* qmbed_mlp;
QMBED_API int qmbed_gpu_mlp_create(int device, int inputs, int outputs, int width, int hidden_layers, uint64_t seed,
                                   qmbed_mlp* out);
QMBED_API int qmbed_gpu_mlp_destroy(qmbed_mlp mlp);
QMBED_API int qmbed_gpu_mlp_parameter_count(qmbed_mlp mlp, uint64_t* count);
QMBED_API int qmbed_gpu_mlp_get_parameters(qmbed_mlp mlp, float* out);
QMBED_API int qmbed_gpu_mlp_set_parameters(qmbed_mlp mlp, const float* in);
/* Input scaling (x - in_mean) / in_std and output scaling y * out_std + out_mean. */
QMBED_API int qmbed_gpu_mlp_set_scaling(qmbed_mlp mlp, const float* in_mean, const float* in_std,
                                        const float* out_mean, const float* out_std);
QMBED_API int qmbed_gpu_mlp_get_scaling(qmbed_mlp mlp, float* in_mean, float* in_std, float* out_mean,
                                        float* out_std);
/* Mean squared error of the unscaled network on n samples (X: n x inputs,
 * Y: n x outputs, row-major) and its gradient for every parameter. */
QMBED_API int qmbed_gpu_mlp_gradients(qmbed_mlp mlp, const float* X, const float* Y, int n, float* grads,
                                      float* loss);
/* Fits the scaling to (X, Y), then trains with Adam (mini-batches, cosine
 * learning-rate decay); loss receives the final full-batch loss (scaled units). */
QMBED_API int qmbed_gpu_mlp_train(qmbed_mlp mlp, const float* X, const float* Y, int n, int epochs, int batch,
                                  float learning_rate, uint64_t seed, float* loss);
QMBED_API int qmbed_gpu_mlp_predict(qmbed_mlp mlp, const float* X, int n, float* Y);

/* ---- Full Lanczos decompositions and thermal Lanczos (FTLM / LTLM) ------ */
/* A device-resident lanczos_ritz decomposition (src/solve/mod.rs:2818-2857;
 * the JSON "lanczos_operator" command, bindings/capi/src/lib.rs:4046-4075):
 * the fully reorthogonalised Krylov basis of op from `initial` (dim complex
 * values), kept in HBM, with its tridiagonal and ascending Ritz system. The
 * recurrence stops after krylov_dimension vectors, when beta <= tolerance, or
 * when the basis spans the operator's whole space. Krylov dimensions above
 * 8192 answer QMBED_STATUS_UNSUPPORTED_BACKEND. */
typedef struct qmbed_lanczos_s* qmbed_lanczos;
QMBED_API int qmbed_gpu_lanczos_create(qmbed_operator op, const double* initial, uint64_t krylov_dimension,
                                       double tolerance, qmbed_lanczos* out);
/* release_lanczos (bindings/capi/src/lib.rs:1874-1886) */
QMBED_API int qmbed_gpu_lanczos_destroy(qmbed_lanczos lanczos);
/* dimension, Krylov length, initial norm, whether the basis is stored real,
 * and the DGKS second passes taken (any pointer may be NULL). */
QMBED_API int qmbed_gpu_lanczos_info(qmbed_lanczos lanczos, uint64_t* dimension, uint64_t* krylov_dimension,
                                     double* initial_norm, int* is_real, uint64_t* second_passes);
/* Ritz values (ascending), column-oriented eigenvectors (vectors[c * m + r] is
 * row r of the eigenvector of values[c]), diagonal and off-diagonal of the
 * tridiagonal (m - 1 values); any pointer may be NULL. */
QMBED_API int qmbed_gpu_lanczos_ritz(qmbed_lanczos lanczos, double* values, double* vectors, double* diagonal,
                                     double* off_diagonal);
/* command_export_lanczos_basis (bindings/capi/src/lib.rs:4293-4310): m x dim complex. */
QMBED_API int qmbed_gpu_lanczos_basis(qmbed_lanczos lanczos, double* basis);
/* LanczosRitzDecomposition::linear_combination (src/solve/mod.rs:2636-2638,
 * linear_combination_qt 3917-3940): out = sum_b coefficients[b] q_b. */
QMBED_API int qmbed_gpu_lanczos_combine(qmbed_lanczos lanczos, const double* coefficients, double* out);
/* LanczosRitzDecomposition::exponential_action (src/solve/mod.rs:2642-2671):
 * out = |v| Q exp(c T) e_1. */
QMBED_API int qmbed_gpu_lanczos_exponential(qmbed_lanczos lanczos, double coefficient_re, double coefficient_im,
                                            double* out);
/* thermal_observable_iteration (src/solve/mod.rs:3858-3872): observables
 * (operators on the same space) projected on the GPU and contracted with the
 * Ritz system; method 0 = FTLM, 1 = LTLM. values[o * n_betas + b] (complex),
 * identity[b]. */
QMBED_API int qmbed_gpu_lanczos_thermal(qmbed_lanczos lanczos, int method, int n_betas, const double* betas,
                                        int n_observables, const qmbed_operator* observables, double* values,
                                        double* identity);
/* LanczosRitzDecomposition::project_thermal_observables for one observable
 * (src/solve/mod.rs:3813-3856), on the GPU: FTLM (method 0) writes the m
 * overlaps <q_i|A|q_0>, LTLM (method 1) the m x m values <q_j|A|q_i> at
 * i * m + j (complex). */
QMBED_API int qmbed_gpu_lanczos_project(qmbed_lanczos lanczos, int method, qmbed_operator observable,
                                        double* matrix_elements);
/* thermal_observable_contraction (src/solve/mod.rs:3785-3806) on host data,
 * with the eigenvector matrix row-major (eigenvectors[r * m + c] = row r of
 * the eigenvector of eigenvalues[c]) as the JSON "lanczos_thermal" command
 * takes it (bindings/capi/src/lib.rs:4214-4237). matrix_elements holds the
 * n_observables projections back to back (m or m * m complex values each). */
QMBED_API int qmbed_gpu_thermal_contraction(int method, int m, const double* eigenvalues, const double* eigenvectors,
                                            int n_observables, const double* matrix_elements, int n_betas,
                                            const double* betas, double* values, double* identity);
/* ftlm_static_iteration / ltlm_static_iteration (src/solve/mod.rs:3543-3568,
 * thermal_lanczos_iteration 3464-3540): log Z and the mean energy at each
 * inverse temperature from one start vector; krylov_out (may be NULL)
 * receives the Krylov length. */
QMBED_API int qmbed_gpu_thermal_iteration(qmbed_operator op, const double* initial, int n_betas, const double* betas,
                                          uint64_t krylov_dimension, double tolerance, double* log_partition,
                                          double* mean_energy, uint64_t* krylov_out);
/* n_vectors FTLM iterations from random start vectors generated on the GPU
 * (Rademacher +-1 entries for real operators, unit phases for complex ones,
 * keyed by seed and the vector index): log_partition and mean_energy
 * [vector][beta], lengths[vector] the Krylov lengths (may be NULL). The
 * reference takes each start vector from its caller; the device sampler has
 * no counterpart there. */
/* Start vector `index` of qmbed_gpu_ftlm_sample for `seed` (dim complex
 * values), so that a run can be repeated from the host. */
QMBED_API int qmbed_gpu_ftlm_start(qmbed_operator op, uint64_t seed, int index, double* out);
QMBED_API int qmbed_gpu_ftlm_sample(qmbed_operator op, int n_vectors, uint64_t seed, int n_betas, const double* betas,
                                    uint64_t krylov_dimension, double tolerance, double* log_partition,
                                    double* mean_energy, int* lengths);

/* ---- Cross-sector action and spectral functions ----------------------- */
/* apply_sector_shift (src/operator/mod.rs:2305-2351): terms (same encoding as
 * qmbed_gpu_operator_create) applied to vectors of `source`, reduced into
 * `target` (same sites and normalisation; momentum, parity and particle
 * number may differ). No Hermiticity or particle checks. */
typedef struct qmbed_shift_s* qmbed_shift;
QMBED_API int qmbed_gpu_shift_create(qmbed_basis source, qmbed_basis target, int n_terms, const int* arity,
                                     const char* symbols, const int* n_couplings, const double* coefficients,
                                     const int* sites, qmbed_shift* out);
QMBED_API int qmbed_gpu_shift_destroy(qmbed_shift shift);
/* Host vectors (interleaved complex): n_input = source dimension, n_output =
 * target dimension, else QMBED_STATUS_DIMENSION_MISMATCH. */
QMBED_API int qmbed_gpu_shift_apply_host(qmbed_shift shift, uint64_t n_input, const double* x, uint64_t n_output,
                                         double* y);
/* Device vectors (interleaved complex FP64), asynchronous on `stream`. */
QMBED_API int qmbed_gpu_shift_apply_device(qmbed_shift shift, const double* x, double* y, void* stream);
/* spectral_function (src/dynamics/mod.rs:964-1021): the probe applied to the
 * source vector (host, n_source complex values), then every eigenpair of the
 * target Hamiltonian when it has at most 128 states, else the Lanczos spectral
 * measure of krylov_dimension steps (src/solve/mod.rs:2886-2907); out[f] =
 * sum_e w_e eta / (pi ((omega_f + reference_energy - E_e)^2 + eta^2)). The
 * probe's target sector must be the Hamiltonian's. */
QMBED_API int qmbed_gpu_spectral_function(qmbed_operator target, qmbed_shift probe, uint64_t n_source,
                                          const double* source, int n_frequencies, const double* frequencies,
                                          double reference_energy, double broadening, uint64_t krylov_dimension,
                                          double tolerance, double* out);

/* deterministic_start (src/solve/mod.rs:729-742): normalised LCG vector. */
QMBED_API int qmbed_gpu_deterministic_start(int device, uint64_t n, uint64_t seed, double* out);

/* ---- JSON boundary: the reference cdylib's exports --------------------- */
/* qmbed_run_json (bindings/capi/src/lib.rs:6089-6106) */
QMBED_API char* qmbed_run_json(const char* request);
/* qmbed_command_json (bindings/capi/src/lib.rs:6120-6137) */
QMBED_API char* qmbed_command_json(const char* request);
/* qmbed_string_free (bindings/capi/src/lib.rs:6290-6296) */
QMBED_API void qmbed_string_free(char* response);
/* qmbed_evolve_model_with_drive_json (bindings/capi/src/lib.rs:6153-6190,
 * 2206-2225, 4695-4746): evolves a registered model's columns under
 * H(t) = H_0 + sum_j c_j(t) H_j with adaptive RK4 step doubling on the GPU;
 * `callback` is int (*)(void* context, double time, {double re, im}* c,
 * size_t count), called at every internal time, 0 on success. */
QMBED_API char* qmbed_evolve_model_with_drive_json(const char* request, void* callback, void* context);
/* qmbed_register_user_basis_{32,64}_json (bindings/capi/src/lib.rs:6192-6282):
 * present for load-time binding; answer an unsupported-backend error. */
QMBED_API char* qmbed_register_user_basis_32_json(const char* request, void* op, void* next_state, void* pre_check,
                                                  void* maps, size_t n_maps);
QMBED_API char* qmbed_register_user_basis_64_json(const char* request, void* op, void* next_state, void* pre_check,
                                                  void* maps, size_t n_maps);

#ifdef __cplusplus
}
#endif

#endif /* QMBED_B200_H */
