// C ABI of libqmbed_b200.so: the typed qmbed_gpu_* API and the JSON
// protocol of the reference cdylib (matrixlab-research/QMBED
// bindings/capi/src/lib.rs). Exceptions never cross the boundary: every
// entry point converts failures into a status code (typed API) or an error
// response (JSON API), like the reference's catch_unwind wrappers
// (lib.rs:6090-6104).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/qmbed_b200.h"
#include "batched.cuh"
#include "chebyshev.cuh"
#include "dense.cuh"
#include "eigsh.cuh"
#include "evolve.cuh"
#include "expm.cuh"
#include "json.hpp"
#include "matrix.cuh"
#include "mlp.cuh"
#include "operator.cuh"
#include "spectrum.cuh"
#include "thermal.cuh"

namespace qmbed {

// Display texts of the reference error variants (src/error.rs:6-35).
void raise(int code, const std::string& detail) {
  std::string text;
  switch (code) {
    case QMBED_INVALID_OPERATOR: text = "invalid or unregistered operator: " + detail; break;
    case QMBED_INVALID_COUPLING: text = "invalid coupling: " + detail; break;
    case QMBED_INVALID_SITE: text = detail; break;
    case QMBED_STATE_NOT_IN_BASIS: text = "state is not represented by this basis"; break;
    case QMBED_INVALID_SECTOR: text = "invalid Hilbert-space sector: " + detail; break;
    case QMBED_INCOMPATIBLE_SYMMETRY: text = "incompatible symmetry request: " + detail; break;
    case QMBED_NON_HERMITIAN: text = "a Hermitian operator is required"; break;
    case QMBED_INVALID_OPTIONS: text = "invalid options: " + detail; break;
    case QMBED_DIMENSION_MISMATCH: text = "dimension mismatch: " + detail; break;
    case QMBED_RANK_DEFICIENT: text = "the supplied vectors are numerically rank deficient"; break;
    case QMBED_UNSUPPORTED_BACKEND: text = "unsupported backend: " + detail; break;
    case QMBED_INTERNAL_STATE: text = "internal state error: " + detail; break;
    case QMBED_CUDA_ERROR: text = "unsupported backend: CUDA error: " + detail; break;
    default: text = detail; break;
  }
  throw Error(code, text);
}

std::atomic<unsigned long long> g_kernel_launches{0};

void count_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

void raise_nonconvergence(size_t iterations, double residual) {
  char buffer[160];
  std::snprintf(buffer, sizeof(buffer), "solver did not converge after %zu iterations; residual=%.6e", iterations,
                residual);
  Error e(QMBED_NON_CONVERGENCE, buffer);
  e.iterations = iterations;
  e.residual = residual;
  throw e;
}

}  // namespace qmbed

using namespace qmbed;

struct qmbed_basis_s {
  std::shared_ptr<SpinBasis> basis;
};

struct qmbed_operator_s {
  std::shared_ptr<SpinOperator> op;
  cudaStream_t stream = nullptr;
  std::unique_ptr<BlockOps> ops;
  std::mutex mu;
  ~qmbed_operator_s() {
    ops.reset();
    if (stream) cudaStreamDestroy(stream);
  }
  BlockOps& block_ops() {
    if (!ops) {
      QMBED_CUDA(cudaSetDevice(op->basis().device()));
      QMBED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      ops = std::make_unique<BlockOps>(op->basis().device(), stream);
    }
    return *ops;
  }
  LinearOperatorView view() {
    BlockOps& b = block_ops();
    SpinOperator* raw = op.get();
    cudaStream_t s = b.stream();
    LinearOperatorView v{raw->dim(), raw->is_real(),
                         [raw, s](int prec, bool cplx, const void* x, void* y) { raw->apply(prec, cplx, x, y, s); }};
    if (raw->supports_block()) {
      v.block_apply = [raw, s](int prec, int nb, const void* z, const void* p, void* out, double alpha, double beta,
                               double gamma) { raw->apply_block(prec, nb, z, p, out, alpha, beta, gamma, s); };
      v.weights = raw->basis().symmetric() ? raw->basis().orbits() : nullptr;
    }
    return v;
  }
};

struct qmbed_lanczos_s {
  LanczosDecomposition d;
  cudaStream_t stream = nullptr;
  std::unique_ptr<BlockOps> ops;
  std::mutex mu;
  ~qmbed_lanczos_s() {
    ops.reset();
    if (stream) cudaStreamDestroy(stream);
  }
  BlockOps& block_ops() {
    if (!ops) {
      QMBED_CUDA(cudaSetDevice(d.device));
      QMBED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      ops = std::make_unique<BlockOps>(d.device, stream);
    }
    return *ops;
  }
};

namespace {

// Host copy of a device column set, widened to interleaved complex.
std::vector<double> lanczos_column_host(const LanczosDecomposition& d, int j) {
  std::vector<double> out(2 * d.n, 0.0);
  if (d.real) {
    std::vector<double> re(d.n);
    QMBED_CUDA(cudaMemcpy(re.data(), d.column(j), d.n * 8, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < d.n; ++i) out[2 * i] = re[i];
  } else {
    QMBED_CUDA(cudaMemcpy(out.data(), d.column(j), d.n * 16, cudaMemcpyDeviceToHost));
  }
  return out;
}

void lanczos_vector_out(qmbed_lanczos_s& l, const std::vector<C64>& c, double* out) {
  DeviceBuffer result(l.d.n * 16);
  lanczos_combine(l.d, c, result.as<double>(), l.block_ops());
  QMBED_CUDA(cudaMemcpy(out, result.get(), l.d.n * 16, cudaMemcpyDeviceToHost));
}

std::vector<double> beta_grid(int n_betas, const double* betas) {
  if (n_betas < 0 || (n_betas > 0 && !betas)) raise(QMBED_INVALID_OPTIONS, "inverse temperatures must be nonempty");
  return std::vector<double>(betas, betas + n_betas);
}

}  // namespace

namespace {

thread_local std::string g_last_error;

// Every entry point leaves the calling thread's current device as it found
// it: the library selects the device of the handle it works on, and an
// embedding host (a framework with its own current device) must not see that.
struct CallerDevice {
  int device = -1;
  CallerDevice() {
    if (cudaGetDevice(&device) != cudaSuccess) {
      device = -1;
      (void)cudaGetLastError();
    }
  }
  ~CallerDevice() {
    int now = -1;
    if (device >= 0 && cudaGetDevice(&now) == cudaSuccess && now != device && cudaSetDevice(device) != cudaSuccess)
      (void)cudaGetLastError();
  }
  CallerDevice(const CallerDevice&) = delete;
  CallerDevice& operator=(const CallerDevice&) = delete;
};

template <typename F>
int guarded(F&& body) {
  CallerDevice restore;
  try {
    body();
    return QMBED_STATUS_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const json::ParseError& e) {
    g_last_error = std::string("invalid options: ") + e.what();
    return QMBED_STATUS_INVALID_OPTIONS;
  } catch (const std::bad_alloc&) {
    g_last_error = "unsupported backend: host allocation failed";
    return QMBED_STATUS_UNSUPPORTED_BACKEND;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal state error: ") + e.what();
    return QMBED_STATUS_INTERNAL_STATE;
  }
}

std::vector<TermDesc> decode_terms(int n_terms, const int* arity, const char* symbols, const int* n_couplings,
                                   const double* coefficients, const int* sites) {
  if (n_terms < 0) raise(QMBED_INVALID_OPTIONS, "negative term count");
  std::vector<TermDesc> terms(static_cast<size_t>(n_terms));
  size_t sc = 0, cc = 0, ss = 0;
  for (int t = 0; t < n_terms; ++t) {
    if (arity[t] <= 0) raise(QMBED_INVALID_OPERATOR, "operator products cannot be empty");
    terms[t].symbols.assign(symbols + sc, symbols + sc + arity[t]);
    sc += static_cast<size_t>(arity[t]);
    for (int c = 0; c < n_couplings[t]; ++c) {
      CouplingDesc coupling;
      coupling.coefficient = C64(coefficients[2 * cc], coefficients[2 * cc + 1]);
      ++cc;
      coupling.sites.assign(sites + ss, sites + ss + arity[t]);
      ss += static_cast<size_t>(arity[t]);
      terms[t].couplings.push_back(std::move(coupling));
    }
  }
  return terms;
}

char* to_c_string(const std::string& s) {
  char* out = static_cast<char*>(std::malloc(s.size() + 1));
  if (!out) return nullptr;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return out;
}

// ---------------------------------------------------------------------------
// JSON protocol (bindings/capi/src/lib.rs:55-2204, 5513-5990)
// ---------------------------------------------------------------------------
using json::Value;

int default_device() {
  const char* env = std::getenv("QMBED_DEVICE");
  return env ? std::atoi(env) : 0;
}

// General lattice maps of the reference's SymmetryRequest
// (bindings/capi/src/lib.rs:3103-3127; LatticeSymmetryMap,
// src/basis/mod.rs:2967-3130) as the built-in chain group. A map moves the
// digit at site i to destinations[i]; one generator step multiplies the orbit
// coefficient by exp(-2 pi i sector / period) (trace_symmetry_orbit,
// src/basis/mod.rs:3455-3538). A translation i -> i + t with gcd(t, L) = 1
// generates every translation, and exp(-2 pi i sector / L) on T^t is the
// built-in momentum k with k t = sector (mod L) (the built-in T moves site i to
// i + 1 with character exp(-2 pi i k / L), src/basis/mod.rs:661-676, 786-790).
// The reflection i -> L-1-i with sector s is the built-in parity (-1)^s, and
// the global spin flip (identity destinations, every local map [1, 0]) with
// sector s is the engine's spin-inversion sector (-1)^s. The reduced vectors,
// gauge (the representative's coefficient) and orbit sizes of both
// constructions agree (GeneralBasis::from_reducer_impl,
// src/basis/mod.rs:4180-4306; spin_symmetry_sector, 715-848). Other maps
// (sublattice translations, partial spin flips, arbitrary permutations) are
// reported as unsupported.
void apply_lattice_maps(const Value& list, SpinBasisDesc& d) {
  const int L = d.sites;
  bool translation = false, reflection = false, inversion = false;
  for (const Value& s : list.items()) {
    const auto& items = s.at("destinations").items();
    if (static_cast<int>(items.size()) != L)
      raise(QMBED_INVALID_OPTIONS, "symmetry map has " + std::to_string(items.size()) + " sites, expected " +
                                       std::to_string(L));
    std::vector<int> dest(L);
    std::vector<char> seen(L, 0);
    for (int i = 0; i < L; ++i) {
      const long long v = items[i].as_int();
      if (v < 0 || v >= L || seen[v]) raise(QMBED_INCOMPATIBLE_SYMMETRY, "symmetry site destinations must be a bijection");
      seen[v] = 1;
      dest[i] = static_cast<int>(v);
    }
    int swaps = 0;
    if (const Value* local = s.find("local_permutations"); local && !local->is_null()) {
      const auto& rows = local->items();
      if (static_cast<int>(rows.size()) != L)
        raise(QMBED_INCOMPATIBLE_SYMMETRY, "every local-state map must be a permutation");
      for (const Value& row : rows) {
        const auto& r = row.items();
        const bool identity = r.size() == 2 && r[0].as_int() == 0 && r[1].as_int() == 1;
        const bool swap = r.size() == 2 && r[0].as_int() == 1 && r[1].as_int() == 0;
        if (!identity && !swap) raise(QMBED_INCOMPATIBLE_SYMMETRY, "every local-state map must be a permutation");
        swaps += swap ? 1 : 0;
      }
    }
    const long long sector = s.at("sector").as_int();
    const int t = dest[0];
    bool is_translation = true, is_reflection = true;
    for (int i = 0; i < L; ++i) {
      is_translation = is_translation && dest[i] == (i + t) % L;
      is_reflection = is_reflection && dest[i] == L - 1 - i;
    }
    if (swaps != 0) {
      // the global spin flip (QuSpin's zblock): every digit swapped, no site moved; period 2
      if (swaps != L || !is_translation || t != 0)
        raise(QMBED_UNSUPPORTED_BACKEND, "local spin maps other than the global spin flip are not supported by the "
                                         "GPU engine");
      if (inversion) raise(QMBED_UNSUPPORTED_BACKEND, "more than one spin-flip generator is not supported by the GPU engine");
      inversion = true;
      d.inversion = ((sector % 2) + 2) % 2 == 0 ? 1 : -1;
      continue;
    }
    if (is_translation && t == 0) continue;  // the identity: period 1, every sector trivial
    if (is_translation) {
      if (std::gcd(t, L) != 1)
        raise(QMBED_UNSUPPORTED_BACKEND, "a translation by " + std::to_string(t) + " of " + std::to_string(L) +
                                             " sites generates a proper subgroup; the GPU engine implements the "
                                             "full translation group");
      if (translation) raise(QMBED_UNSUPPORTED_BACKEND, "more than one translation generator is not supported by the GPU engine");
      translation = true;
      long long inverse = 1;  // t^-1 mod L by trial: L is at most 128
      while ((inverse * t) % L != 1 % L) ++inverse;
      const long long canonical = ((sector % L) + L) % L;
      d.has_momentum = 1;
      d.momentum = static_cast<int>((canonical * inverse) % L);
    } else if (is_reflection) {
      if (reflection) raise(QMBED_UNSUPPORTED_BACKEND, "more than one reflection generator is not supported by the GPU engine");
      reflection = true;
      d.parity = ((sector % 2) + 2) % 2 == 0 ? 1 : -1;
    } else {
      raise(QMBED_UNSUPPORTED_BACKEND,
            "lattice maps other than chain translations and the reflection site -> L-1-site are not supported "
            "by the GPU engine");
    }
  }
}

// A spin basis request as the engine builds it. The reference's `reverse`
// flag (bindings/capi/src/lib.rs:2849-2905, 3412-3423) reverses the public
// row order and, for lattice-map sectors, takes the maximum orbit state as
// the representative. Bitwise complement (the global spin flip C) reverses
// the order of integers and commutes with every site permutation, so that
// basis is, row for row and phase for phase, the complement of the ordinary
// (minimum-representative, ascending) sector with up' = L - up. The engine
// builds that sector (`flipped`) and acts with C H C: its local products
// follow flip_terms below, and every vector, matrix entry and eigenvector
// keeps the reference's row order without a permutation.
struct BasisRequest {
  SpinBasisDesc desc;
  bool flipped = false;
};

BasisRequest parse_basis(const Value& b) {
  const std::string kind = b.at("kind").as_string();
  if (kind != "spin")
    raise(QMBED_UNSUPPORTED_BACKEND, "the GPU engine implements spin-1/2 chain bases; `" + kind + "` is not supported");
  BasisRequest r;
  SpinBasisDesc& d = r.desc;
  d = SpinBasisDesc{};
  d.sites = static_cast<int>(b.at("sites").as_int());
  if (b.has("spin_twice") && b.at("spin_twice").as_int() != 1)
    raise(QMBED_UNSUPPORTED_BACKEND, "the GPU engine implements spin one half (spin_twice = 1)");
  if (b.has("up") && b.has("up_sectors"))
    raise(QMBED_INVALID_OPTIONS, "spin basis accepts either up or up_sectors, not both");
  d.up = b.has("up") ? static_cast<int>(b.at("up").as_int()) : -1;
  if (b.has("up_sectors")) {
    const auto& sectors = b.at("up_sectors").items();
    if (sectors.size() != 1) raise(QMBED_UNSUPPORTED_BACKEND, "unions of magnetisation sectors are not supported");
    d.up = static_cast<int>(sectors[0].as_int());
  }
  d.has_momentum = b.has("momentum") ? 1 : 0;
  d.momentum = d.has_momentum ? static_cast<int>(b.at("momentum").as_int()) : 0;
  d.parity = b.has("parity") ? static_cast<int>(b.at("parity").as_int()) : 0;
  const bool built_in = d.has_momentum || d.parity;
  d.normalization = (b.has("pauli") && b.at("pauli").as_bool()) ? kPauliCartesian : kAngularMomentum;
  if (b.has("normalization")) {
    const std::string n = b.at("normalization").as_string();
    if (n == "angular_momentum") d.normalization = kAngularMomentum;
    else if (n == "pauli") d.normalization = kPauli;
    else if (n == "pauli_cartesian") d.normalization = kPauliCartesian;
    else raise(QMBED_INVALID_OPTIONS, "unknown spin normalization `" + n + "`");
  }
  if (b.has("symmetries") && !b.at("symmetries").items().empty()) {
    if (built_in) raise(QMBED_INVALID_OPTIONS, "built-in and general spin symmetries cannot be mixed");
    if (d.sites <= 0) raise(QMBED_INVALID_SECTOR, "symmetry sectors require at least one site");
    apply_lattice_maps(b.at("symmetries"), d);
  }
  if (b.has("matrix_symmetry"))
    raise(QMBED_INVALID_OPTIONS, "matrix-valued symmetry sectors materialize as projected operator models");
  if (b.has("reverse") && b.at("reverse").as_bool()) {
    if (built_in)
      raise(QMBED_UNSUPPORTED_BACKEND, "the reversed order of built-in momentum or parity sectors is not supported by "
                                       "the GPU engine (send the sector as lattice maps)");
    if (d.up > d.sites) raise(QMBED_INVALID_SECTOR, "particle count exceeds site count");
    if (d.up >= 0) d.up = d.sites - d.up;
    r.flipped = true;
  }
  return r;
}

// typed_local_operator (bindings/capi/src/lib.rs:6053-6071)
char local_symbol(const std::string& name) {
  if (name == "identity") return 'I';
  if (name == "number") return 'n';
  if (name == "z") return 'z';
  if (name == "raising") return '+';
  if (name == "lowering") return '-';
  if (name == "x") return 'x';
  if (name == "y") return 'y';
  if (name.rfind("custom:", 0) == 0 && name.size() == 8) return name[7];
  raise(QMBED_INVALID_OPERATOR, name);
}

std::vector<TermDesc> parse_terms(const Value& terms, C64 scale = C64(1.0, 0.0)) {
  std::vector<TermDesc> out;
  for (const Value& t : terms.items()) {
    TermDesc term;
    for (const Value& name : t.at("product").at("local").items()) term.symbols.push_back(local_symbol(name.as_string()));
    if (term.symbols.empty()) raise(QMBED_INVALID_OPERATOR, "operator products cannot be empty");
    for (const Value& c : t.at("couplings").items()) {
      const auto& coef = c.at("coefficient").items();
      if (coef.size() != 2) raise(QMBED_INVALID_OPTIONS, "coefficients are [re, im] pairs");
      CouplingDesc coupling;
      coupling.coefficient = scale * C64(coef[0].as_double(), coef[1].as_double());
      for (const Value& s : c.at("sites").items()) {
        const long long site = s.as_int();
        if (site < 0) raise(QMBED_INVALID_OPTIONS, "sites are non-negative integers");
        coupling.sites.push_back(static_cast<int>(site));
      }
      term.couplings.push_back(std::move(coupling));
    }
    out.push_back(std::move(term));
  }
  return out;
}

// Spin-flip image C P C of one local product: C z C = -z, C S+ C = S-,
// C S- C = S+, C x C = x and C y C = -y in every normalisation of spin one
// half. Other symbols pass through and are rejected when the operator is built.
std::vector<TermDesc> flip_terms(std::vector<TermDesc> terms) {
  for (TermDesc& t : terms) {
    double sign = 1.0;
    for (char& c : t.symbols) {
      if (c == 'z' || c == 'y') sign = -sign;
      else if (c == '+') c = '-';
      else if (c == '-') c = '+';
    }
    for (auto& coupling : t.couplings) coupling.coefficient *= sign;
  }
  return terms;
}

// The site labels a frontend uses for one model: the reference's
// site_permutation (OperatorSpec::with_site_permutation,
// src/operator/mod.rs:264-300, applied to terms and components by
// EdModel::with_site_permutation and to later term requests by
// prepare_terms, src/interop.rs:682-707, 1285-1296), followed by the spin flip
// of a reversed basis.
struct SiteConvention {
  std::vector<int> permutation;  // empty: identity
  bool flipped = false;

  bool same_sites(const SiteConvention& o) const { return permutation == o.permutation; }

  std::vector<TermDesc> prepare(std::vector<TermDesc> terms) const {
    if (!permutation.empty())
      for (TermDesc& t : terms)
        for (auto& coupling : t.couplings)
          for (int& site : coupling.sites) {
            if (site >= static_cast<int>(permutation.size()))
              raise(QMBED_INVALID_SITE, "site " + std::to_string(site) + " is outside a lattice with " +
                                            std::to_string(permutation.size()) + " sites");
            site = permutation[site];
          }
    return flipped ? flip_terms(std::move(terms)) : terms;
  }
};

// validate_site_permutation (src/interop.rs:1328-1344)
SiteConvention parse_convention(const Value& request, bool flipped) {
  SiteConvention c;
  c.flipped = flipped;
  if (const Value* p = request.find("site_permutation"); p && !p->is_null()) {
    const auto& items = p->items();
    const long long n = static_cast<long long>(items.size());
    for (const Value& v : items) {
      const long long site = v.as_int();
      if (site < 0) raise(QMBED_INVALID_OPTIONS, "site permutation entries are non-negative integers");
      if (site >= n)
        raise(QMBED_INVALID_SITE, "site " + std::to_string(site) + " is outside a lattice with " + std::to_string(n) +
                                      " sites");
    }
    std::vector<char> seen(items.size(), 0);
    for (const Value& v : items) {
      const long long site = v.as_int();
      if (seen[site]) raise(QMBED_INVALID_OPTIONS, "site permutation must be bijective");
      seen[site] = 1;
      c.permutation.push_back(static_cast<int>(site));
    }
  }
  return c;
}

OperatorChecks parse_checks(const Value& request) {
  OperatorChecks checks;
  if (const Value* c = request.find("checks")) {
    if (c->has("hermiticity")) checks.hermiticity = c->at("hermiticity").as_bool();
    if (c->has("particle_conservation")) checks.particle_conservation = c->at("particle_conservation").as_bool();
  }
  return checks;
}

int parse_storage(const Value& request) {
  if (!request.has("format")) return kStoragePacked;
  const std::string f = request.at("format").as_string();
  if (f == "matrix_free") return kStorageMatrixFree;
  if (f == "dense" || f == "csc" || f == "csr" || f == "dia") return kStoragePacked;
  raise(QMBED_INVALID_OPTIONS, "unknown storage format `" + f + "`");
}

struct SolverRequest {
  EigshOptions options;
  bool eigenvectors = false;
  int mode = kModePlainFP64;
  std::vector<std::vector<C64>> initial;
};

std::vector<C64> parse_vector(const Value& v) {
  std::vector<C64> out;
  for (const Value& pair : v.items()) {
    const auto& p = pair.items();
    if (p.size() != 2) raise(QMBED_INVALID_OPTIONS, "vector entries are [re, im] pairs");
    out.emplace_back(p[0].as_double(), p[1].as_double());
  }
  return out;
}

SolverRequest parse_solver(const Value& s) {
  SolverRequest r;
  r.options.eigenpairs = static_cast<size_t>(s.at("eigenpairs").as_int());
  const std::string kind = s.at("target").at("kind").as_string();
  if (kind == "smallest_algebraic") r.options.target = kSmallestAlgebraic;
  else if (kind == "largest_algebraic") r.options.target = kLargestAlgebraic;
  else if (kind == "smallest_magnitude") r.options.target = kSmallestMagnitude;
  else if (kind == "largest_magnitude") r.options.target = kLargestMagnitude;
  else if (kind == "both_ends") r.options.target = kBothEnds;
  else if (kind == "shift") {
    r.options.target = kShift;
    r.options.shift = s.at("target").at("value").as_double();
  } else {
    raise(QMBED_INVALID_OPTIONS, "unknown spectrum target `" + kind + "`");
  }
  if (s.has("krylov_dimension")) r.options.krylov_dimension = static_cast<size_t>(s.at("krylov_dimension").as_int());
  if (s.has("tolerance")) r.options.tolerance = s.at("tolerance").as_double();
  if (s.has("max_iterations")) r.options.max_iterations = static_cast<size_t>(s.at("max_iterations").as_int());
  if (s.has("seed")) r.options.seed = static_cast<uint64_t>(s.at("seed").as_int());
  if (s.has("eigenvectors")) r.eigenvectors = s.at("eigenvectors").as_bool();
  if (s.has("initial_vector")) r.initial.push_back(parse_vector(s.at("initial_vector")));
  else if (s.has("v0")) r.initial.push_back(parse_vector(s.at("v0")));
  if (s.has("precision")) {
    const std::string p = s.at("precision").as_string();
    if (p == "mixed") r.mode = kModeMixed;
    else if (p == "filtered") r.mode = kModeFiltered;
    else if (p != "fp64") raise(QMBED_INVALID_OPTIONS, "precision must be `fp64`, `mixed` or `filtered`");
  }
  return r;
}

Value complex_pair(C64 v) {
  Value p = Value::array();
  p.push(Value::number(v.real()));
  p.push(Value::number(v.imag()));
  return p;
}

Value vectors_value(const std::vector<double>& host, uint64_t dim, size_t count) {
  Value vs = Value::array();
  for (size_t k = 0; k < count; ++k) {
    Value v = Value::array();
    for (uint64_t i = 0; i < dim; ++i) v.push(complex_pair(C64(host[2 * (k * dim + i)], host[2 * (k * dim + i) + 1])));
    vs.push(std::move(v));
  }
  return vs;
}

// Runs eigsh and returns the SolveResult / Eigensystem JSON fields.
Value solve_view(const LinearOperatorView& view, BlockOps& ops, const SolverRequest& request, bool tagged) {
  std::vector<double> initial;
  for (const auto& v : request.initial) {
    if (v.size() != view.dim) raise(QMBED_DIMENSION_MISMATCH, "eigsh initial vector does not match the operator");
    for (const C64& x : v) {
      initial.push_back(x.real());
      initial.push_back(x.imag());
    }
  }
  EigshOptions options = request.options;
  options.want_vectors = request.eigenvectors;
  EigshResult r = eigsh(view, options, initial.data(), static_cast<int>(request.initial.size()), request.mode, ops);
  Value out = Value::object();
  if (tagged) out.set("kind", Value::string("eigensystem"));
  const uint64_t dim = view.dim;
  out.set("dimension", Value::integer(static_cast<long long>(dim)));
  Value values = Value::array(), residuals = Value::array();
  for (double v : r.eigenvalues) values.push(Value::number(v));
  for (double v : r.residuals) residuals.push(Value::number(v));
  out.set("eigenvalues", std::move(values));
  out.set("residuals", std::move(residuals));
  out.set("iterations", Value::integer(static_cast<long long>(r.iterations)));
  out.set("converged", Value::boolean(r.converged));
  if (request.eigenvectors) {
    const size_t k = r.eigenvalues.size();
    std::vector<double> host(2 * k * dim, 0.0);
    if (r.complex_vectors) {
      QMBED_CUDA(cudaMemcpy(host.data(), r.vectors.get(), host.size() * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<double> real(k * dim);
      QMBED_CUDA(cudaMemcpy(real.data(), r.vectors.get(), real.size() * 8, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < real.size(); ++i) host[2 * i] = real[i];
    }
    out.set("eigenvectors", vectors_value(host, dim, k));
  }
  return out;
}

Value solve(qmbed_operator_s& handle, const SolverRequest& request, bool tagged) {
  std::lock_guard<std::mutex> lock(handle.mu);
  return solve_view(handle.view(), handle.block_ops(), request, tagged);
}

std::shared_ptr<qmbed_operator_s> make_operator(std::shared_ptr<SpinBasis> basis, const std::vector<TermDesc>& terms,
                                                const OperatorChecks& checks, int storage) {
  auto h = std::make_shared<qmbed_operator_s>();
  h->op = std::make_shared<SpinOperator>(std::move(basis), terms, checks, storage);
  return h;
}

// The adjoint of local products: each product reversed with S+ <-> S- and the
// coupling sites in the same reversed order, coefficients conjugated
// (z, x, y and the identity are Hermitian).
std::vector<TermDesc> adjoint_terms(const std::vector<TermDesc>& terms) {
  std::vector<TermDesc> out;
  for (const TermDesc& t : terms) {
    TermDesc a;
    a.symbols.assign(t.symbols.rbegin(), t.symbols.rend());
    for (char& c : a.symbols) c = c == '+' ? '-' : (c == '-' ? '+' : c);
    for (const CouplingDesc& coupling : t.couplings) {
      CouplingDesc d;
      d.coefficient = std::conj(coupling.coefficient);
      d.sites.assign(coupling.sites.rbegin(), coupling.sites.rend());
      a.couplings.push_back(std::move(d));
    }
    out.push_back(std::move(a));
  }
  return out;
}

// OperatorActionRequest (bindings/capi/src/lib.rs:937-945). Conjugate and
// transpose are applied as conj(H conj(x)) and conj(H^dagger conj(x)).
enum class Action { kNormal, kTranspose, kConjugate, kAdjoint };

Action parse_action(const Value& owner) {
  if (!owner.has("action")) return Action::kNormal;
  const std::string a = owner.at("action").as_string();
  if (a == "normal") return Action::kNormal;
  if (a == "transpose") return Action::kTranspose;
  if (a == "conjugate") return Action::kConjugate;
  if (a == "adjoint") return Action::kAdjoint;
  raise(QMBED_INVALID_OPTIONS, "unknown operator action `" + a + "`");
}

bool uses_adjoint(Action a) { return a == Action::kTranspose || a == Action::kAdjoint; }
bool conjugates(Action a) { return a == Action::kTranspose || a == Action::kConjugate; }

struct Component {
  std::string name;
  std::vector<TermDesc> terms;
  bool has_default;
  C64 default_value;
};

struct Model {
  uint64_t id = 0;  // registry id (never reused), 0 for unregistered models
  std::shared_ptr<SpinBasis> basis;
  SiteConvention convention;
  std::vector<TermDesc> terms;
  std::vector<Component> components;
  OperatorChecks checks;
  std::mutex mu;
  std::map<std::string, std::shared_ptr<qmbed_operator_s>> cache;  // parameters+storage -> operator

  // The model's terms with every component scaled by its parameter value
  // (supplied, else the default); `key` receives the parameter values.
  std::vector<TermDesc> resolved_terms(const Value* parameters, std::string& key) const {
    std::map<std::string, C64> values;
    if (parameters && parameters->is_object())
      for (auto& kv : parameters->members()) {
        bool known = false;
        for (auto& c : components) known = known || c.name == kv.first;
        if (!known) raise(QMBED_INVALID_OPTIONS, "unknown operator parameter \"" + kv.first + "\"");
        const auto& p = kv.second.items();
        values[kv.first] = C64(p.at(0).as_double(), p.at(1).as_double());
      }
    std::vector<TermDesc> all = terms;
    for (auto& c : components) {
      C64 v;
      auto it = values.find(c.name);
      if (it != values.end()) v = it->second;
      else if (c.has_default) v = c.default_value;
      else raise(QMBED_INVALID_OPTIONS, "operator parameter \"" + c.name + "\" has no default and was not supplied");
      char buffer[96];
      std::snprintf(buffer, sizeof(buffer), "|%.17g,%.17g", v.real(), v.imag());
      key += buffer;
      for (const TermDesc& t : c.terms) {
        TermDesc scaled = t;
        for (auto& coupling : scaled.couplings) coupling.coefficient *= v;
        all.push_back(std::move(scaled));
      }
    }
    return all;
  }

  // One operator per distinct key, built on first use.
  std::shared_ptr<qmbed_operator_s> cached(const std::string& key, const std::vector<TermDesc>& all, OperatorChecks c,
                                           int storage) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    auto op = make_operator(basis, all, c, storage);
    cache[key] = op;
    return op;
  }

  // H (normal, conjugate) or H^dagger (adjoint, transpose) at the parameters
  std::shared_ptr<qmbed_operator_s> materialize_action(const Value* parameters, int storage, Action action) {
    if (!uses_adjoint(action)) return materialize(parameters, storage, false);
    std::string key = "adjoint|" + std::to_string(storage);
    const std::vector<TermDesc> all = adjoint_terms(resolved_terms(parameters, key));
    OperatorChecks c = checks;
    c.hermiticity = false;
    return cached(key, all, c, storage);
  }

  std::shared_ptr<qmbed_operator_s> materialize(const Value* parameters, int storage, bool hermitian_check) {
    std::string key = std::to_string(storage) + (hermitian_check ? "h" : "n");
    const std::vector<TermDesc> all = resolved_terms(parameters, key);
    OperatorChecks c = checks;
    c.hermiticity = hermitian_check && checks.hermiticity;
    return cached(key, all, c, storage);
  }
};

// An operator model given by explicit matrix entries: create_operator_model
// with a static operator and neither components nor a basis
// (build_operator_model, bindings/capi/src/lib.rs:5605-5622). Its handle
// shares the model handle sequence.
struct MatrixModel {
  std::shared_ptr<CsrMatrix> matrix;
  cudaStream_t stream = nullptr;
  std::unique_ptr<BlockOps> ops;
  std::mutex mu;
  ~MatrixModel() {
    ops.reset();
    if (stream) cudaStreamDestroy(stream);
  }
  BlockOps& block_ops() {
    if (!ops) {
      QMBED_CUDA(cudaSetDevice(matrix->device()));
      QMBED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      ops = std::make_unique<BlockOps>(matrix->device(), stream);
    }
    return *ops;
  }
  LinearOperatorView view() {
    BlockOps& b = block_ops();
    const CsrMatrix* raw = matrix.get();
    cudaStream_t s = b.stream();
    return LinearOperatorView{raw->dim(), raw->is_real(), [raw, s](int prec, bool cplx, const void* x, void* y) {
                                raw->apply(prec, cplx, x, y, s);
                              }};
  }
};

struct ExpmEntry {
  std::shared_ptr<qmbed_operator_s> op;
  std::shared_ptr<MatrixModel> matrix;  // set instead of `op` for explicit-matrix models
  ExpmPlan plan;
};

std::mutex g_registry_mu;
std::map<uint64_t, std::shared_ptr<Model>> g_models;
std::map<uint64_t, std::shared_ptr<ExpmEntry>> g_expm;
std::atomic<uint64_t> g_next_model{1}, g_next_expm{1};
std::map<uint64_t, std::shared_ptr<qmbed_lanczos_s>> g_lanczos;
std::atomic<uint64_t> g_next_lanczos{1};

uint64_t parse_handle(const std::string& text, const char* what) {
  char* end = nullptr;
  const unsigned long long value = std::strtoull(text.c_str(), &end, 10);
  if (text.empty() || !end || *end != '\0' || value == 0)
    raise(QMBED_INVALID_OPTIONS, std::string(what) + " handle \"" + text + "\" is not a positive integer");
  return value;
}

std::map<uint64_t, std::shared_ptr<MatrixModel>> g_matrix_models;

// The explicit-matrix model behind a model handle, or null for a term model.
std::shared_ptr<MatrixModel> matrix_model(const std::string& text) {
  const uint64_t id = parse_handle(text, "model");
  std::lock_guard<std::mutex> lock(g_registry_mu);
  auto it = g_matrix_models.find(id);
  return it == g_matrix_models.end() ? nullptr : it->second;
}

// MatrixRequest (bindings/capi/src/lib.rs:744-754): shape and entries.
std::shared_ptr<CsrMatrix> parse_matrix(const Value& m) {
  const auto& shape = m.at("shape").items();
  if (shape.size() != 2) raise(QMBED_INVALID_OPTIONS, "matrix shape is a [rows, columns] pair");
  const long long rows = shape[0].as_int(), cols = shape[1].as_int();
  if (rows < 0 || cols < 0) raise(QMBED_INVALID_OPTIONS, "matrix shape entries are non-negative");
  if (rows != cols) raise(QMBED_DIMENSION_MISMATCH, "an operator model requires a square matrix");
  std::vector<uint64_t> r, c;
  std::vector<C64> v;
  for (const Value& e : m.at("entries").items()) {
    const long long row = e.at("row").as_int(), column = e.at("column").as_int();
    if (row < 0 || column < 0) raise(QMBED_INVALID_OPTIONS, "matrix entry indices are non-negative");
    const auto& value = e.at("value").items();
    if (value.size() != 2) raise(QMBED_INVALID_OPTIONS, "matrix values are [re, im] pairs");
    r.push_back(static_cast<uint64_t>(row));
    c.push_back(static_cast<uint64_t>(column));
    v.emplace_back(value[0].as_double(), value[1].as_double());
  }
  return std::make_shared<CsrMatrix>(default_device(), static_cast<uint64_t>(rows), r, c, v);
}

std::shared_ptr<Model> registered_model(const std::string& text) {
  const uint64_t id = parse_handle(text, "model");
  std::lock_guard<std::mutex> lock(g_registry_mu);
  auto it = g_models.find(id);
  if (it == g_models.end()) raise(QMBED_INVALID_OPTIONS, "model handle " + text + " is not registered");
  return it->second;
}

std::shared_ptr<ExpmEntry> registered_expm(const std::string& text) {
  const uint64_t id = parse_handle(text, "exponential-action");
  std::lock_guard<std::mutex> lock(g_registry_mu);
  auto it = g_expm.find(id);
  if (it == g_expm.end()) raise(QMBED_INVALID_OPTIONS, "exponential-action handle " + text + " is not registered");
  return it->second;
}

// parse_lanczos_handle / registered_lanczos (bindings/capi/src/lib.rs:1672-1872):
// "lanczos:<positive integer>".
uint64_t parse_lanczos_handle(const std::string& text) {
  if (text.rfind("lanczos:", 0) != 0)
    raise(QMBED_INVALID_OPTIONS, "Lanczos handle \"" + text + "\" does not use the lanczos: prefix");
  const std::string digits = text.substr(8);
  char* end = nullptr;
  const unsigned long long value = std::strtoull(digits.c_str(), &end, 10);
  if (digits.empty() || !end || *end != '\0') raise(QMBED_INVALID_OPTIONS, "Lanczos handle \"" + text + "\" is invalid");
  return value;
}

std::shared_ptr<qmbed_lanczos_s> registered_lanczos(const std::string& text) {
  const uint64_t id = parse_lanczos_handle(text);
  std::lock_guard<std::mutex> lock(g_registry_mu);
  auto it = g_lanczos.find(id);
  if (it == g_lanczos.end()) raise(QMBED_INVALID_OPTIONS, "Lanczos handle " + text + " is not registered");
  return it->second;
}

std::shared_ptr<Model> build_model(const Value& request) {
  auto model = std::make_shared<Model>();
  const BasisRequest basis = parse_basis(request.at("basis"));
  model->convention = parse_convention(request, basis.flipped);
  model->terms = model->convention.prepare(parse_terms(request.at("terms")));
  model->checks = parse_checks(request);
  if (const Value* comps = request.find("components"))
    if (comps->is_array())
      for (const Value& c : comps->items()) {
        Component comp;
        comp.name = c.at("name").as_string();
        comp.terms = model->convention.prepare(parse_terms(c.at("terms")));
        comp.has_default = c.has("default");
        if (comp.has_default) {
          const auto& d = c.at("default").items();
          comp.default_value = C64(d.at(0).as_double(), d.at(1).as_double());
        }
        model->components.push_back(std::move(comp));
      }
  model->basis = std::make_shared<SpinBasis>(basis.desc, default_device());
  return model;
}

std::vector<std::vector<C64>> parse_vectors(const Value& v) {
  std::vector<std::vector<C64>> out;
  for (const Value& vec : v.items()) out.push_back(parse_vector(vec));
  return out;
}

// The operator applied to host columns, one GPU application per column.
std::vector<std::vector<C64>> apply_columns(const LinearOperatorView& view, BlockOps& ops,
                                            const std::vector<std::vector<C64>>& vectors, const char* mismatch) {
  const uint64_t dim = view.dim;
  DeviceBuffer x(std::max<uint64_t>(dim, 1) * 16), y(std::max<uint64_t>(dim, 1) * 16);
  std::vector<double> host(2 * dim);
  std::vector<std::vector<C64>> out;
  out.reserve(vectors.size());
  for (const auto& v : vectors) {
    if (v.size() != dim) raise(QMBED_DIMENSION_MISMATCH, mismatch);
    for (uint64_t i = 0; i < dim; ++i) {
      host[2 * i] = v[i].real();
      host[2 * i + 1] = v[i].imag();
    }
    QMBED_CUDA(cudaMemcpyAsync(x.get(), host.data(), 16 * dim, cudaMemcpyHostToDevice, ops.stream()));
    view.apply(64, true, x.get(), y.get());
    QMBED_CUDA(cudaMemcpyAsync(host.data(), y.get(), 16 * dim, cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
    std::vector<C64> r(dim);
    for (uint64_t i = 0; i < dim; ++i) r[i] = C64(host[2 * i], host[2 * i + 1]);
    out.push_back(std::move(r));
  }
  return out;
}

std::vector<std::vector<C64>> apply_columns(qmbed_operator_s& handle, const std::vector<std::vector<C64>>& vectors,
                                            const char* mismatch) {
  std::lock_guard<std::mutex> lock(handle.mu);
  return apply_columns(handle.view(), handle.block_ops(), vectors, mismatch);
}

Value vectors_result(const std::vector<std::vector<C64>>& applied, uint64_t dim) {
  Value out = Value::object();
  out.set("kind", Value::string("vectors"));
  out.set("dimension", Value::integer(static_cast<long long>(dim)));
  Value vs = Value::array();
  for (const auto& v : applied) {
    Value r = Value::array();
    for (const C64& e : v) r.push(complex_pair(e));
    vs.push(std::move(r));
  }
  out.set("vectors", std::move(vs));
  return out;
}

Value apply_vectors(qmbed_operator_s& handle, const std::vector<std::vector<C64>>& vectors) {
  const auto applied = apply_columns(handle, vectors, "vector length does not match the model dimension");
  return vectors_result(applied, handle.op->dim());
}

// A x, or conj(A conj(x)) for the conjugating actions.
Value apply_with_action(qmbed_operator_s& handle, std::vector<std::vector<C64>> vectors, bool conjugate) {
  if (!conjugate) return apply_vectors(handle, vectors);
  for (auto& v : vectors)
    for (C64& x : v) x = std::conj(x);
  auto applied = apply_columns(handle, vectors, "vector length does not match the model dimension");
  for (auto& v : applied)
    for (C64& x : v) x = std::conj(x);
  return vectors_result(applied, handle.op->dim());
}

// inner (src/measure/mod.rs:68-73): conjugate-linear in the left argument
C64 inner(const std::vector<C64>& left, const std::vector<C64>& right) {
  C64 sum(0.0, 0.0);
  for (size_t i = 0; i < left.size() && i < right.size(); ++i) sum += std::conj(left[i]) * right[i];
  return sum;
}

Value measurements_value(std::vector<long long> shape, const std::vector<C64>& values) {
  Value out = Value::object();
  out.set("kind", Value::string("measurements"));
  Value s = Value::array();
  for (long long n : shape) s.push(Value::integer(n));
  out.set("shape", std::move(s));
  Value v = Value::array();
  for (const C64& x : values) v.push(complex_pair(x));
  out.set("values", std::move(v));
  return out;
}

// command_matrix_elements (bindings/capi/src/lib.rs:4362-4396) with
// matrix_element (src/measure/mod.rs:101-115): <left| H |right> for every
// pair, or for matching pairs when `diagonal`.
Value matrix_elements(Model& model, const Value& request) {
  const auto left = parse_vectors(request.at("left_vectors"));
  const auto right = parse_vectors(request.at("right_vectors"));
  const bool diagonal = request.has("diagonal") && request.at("diagonal").as_bool();
  if (diagonal && left.size() != right.size())
    raise(QMBED_DIMENSION_MISMATCH, "diagonal matrix elements require equal vector batches");
  auto op = model.materialize(request.find("parameters"), kStoragePacked, false);
  const char* mismatch = "matrix-element vectors do not match the operator shape";
  for (const auto& l : left)
    if (l.size() != op->op->dim()) raise(QMBED_DIMENSION_MISMATCH, mismatch);
  const auto applied = apply_columns(*op, right, mismatch);
  std::vector<C64> values;
  if (diagonal) {
    for (size_t i = 0; i < left.size(); ++i) values.push_back(inner(left[i], applied[i]));
    return measurements_value({static_cast<long long>(left.size())}, values);
  }
  for (const auto& l : left)
    for (const auto& a : applied) values.push_back(inner(l, a));
  return measurements_value({static_cast<long long>(left.size()), static_cast<long long>(right.size())}, values);
}

// command_measure_model (bindings/capi/src/lib.rs:4398-4432): per sample,
// expectation <s|H|s> and raw fluctuation <s|H^2|s> - <s|H|s>^2 of a pure
// state (src/measure/mod.rs:117-175), or Tr(rho H) and Tr(rho H^2) - Tr(rho H)^2
// of a row-major density matrix (1336-1390); no normalisation is imposed.
Value measure(Model& model, const Value& request) {
  const std::string what = request.at("measurement").as_string();
  const bool fluctuation = what == "quantum_fluctuation";
  if (!fluctuation && what != "expectation")
    raise(QMBED_INVALID_OPTIONS, "measurement must be `expectation` or `quantum_fluctuation`");
  std::vector<C64> values;
  for (const Value& sample : request.at("samples").items()) {
    const std::string kind = sample.at("kind").as_string();
    if (kind != "pure" && kind != "density") raise(QMBED_INVALID_OPTIONS, "measurement samples are `pure` or `density`");
    const auto state = parse_vector(sample.at("values"));
    auto op = model.materialize(sample.find("parameters"), kStoragePacked, false);
    const uint64_t dim = op->op->dim();
    if (kind == "pure") {
      const char* mismatch = fluctuation ? "raw quantum fluctuation requires a square operator matching the state"
                                         : "matrix-element vectors do not match the operator shape";
      const auto once = apply_columns(*op, {state}, mismatch);
      const C64 mean = inner(state, once[0]);
      if (!fluctuation) {
        values.push_back(mean);
        continue;
      }
      const auto twice = apply_columns(*op, once, mismatch);
      values.push_back(inner(state, twice[0]) - mean * mean);
      continue;
    }
    if (state.size() != dim * dim)
      raise(QMBED_DIMENSION_MISMATCH, fluctuation ? "density fluctuation requires a square operator and matching density"
                                                  : "density expectation requires a square operator and matching density");
    std::vector<std::vector<C64>> columns(dim, std::vector<C64>(dim));
    for (uint64_t r = 0; r < dim; ++r)
      for (uint64_t c = 0; c < dim; ++c) columns[c][r] = state[r * dim + c];
    const auto once = apply_columns(*op, columns, "density expectation requires a square operator and matching density");
    C64 mean(0.0, 0.0);
    for (uint64_t c = 0; c < dim; ++c) mean += once[c][c];
    if (!fluctuation) {
      values.push_back(mean);
      continue;
    }
    const auto twice = apply_columns(*op, once, "density fluctuation requires a square operator and matching density");
    C64 second(0.0, 0.0);
    for (uint64_t c = 0; c < dim; ++c) second += twice[c][c];
    values.push_back(second - mean * mean);
  }
  return measurements_value({static_cast<long long>(values.size())}, values);
}

Value run_request(const Value& request) {
  auto model = build_model(request);
  auto op = model->materialize(nullptr, parse_storage(request), true);
  return solve(*op, parse_solver(request.at("solver")), false);
}

Value describe_basis(const Value& request) {
  const BasisRequest request_basis = parse_basis(request.at("basis"));
  SpinBasis basis(request_basis.desc, default_device());
  const uint64_t n = basis.dim();
  std::vector<uint64_t> lo(n), hi(n);
  basis.copy_states(0, n, lo.data(), hi.data(), nullptr);
  if (request_basis.flipped) {  // the reversed basis lists the complements of the engine's states
    const int L = request_basis.desc.sites;
    const uint64_t lo_mask = L >= 64 ? ~0ull : (1ull << L) - 1;
    const uint64_t hi_mask = L >= 128 ? ~0ull : (L > 64 ? (1ull << (L - 64)) - 1 : 0ull);
    for (uint64_t i = 0; i < n; ++i) {
      lo[i] = ~lo[i] & lo_mask;
      hi[i] = ~hi[i] & hi_mask;
    }
  }
  Value out = Value::object();
  out.set("kind", Value::string("basis"));
  out.set("dimension", Value::integer(static_cast<long long>(n)));
  Value states = Value::array();
  for (uint64_t i = 0; i < n; ++i) {
    unsigned __int128 s = (static_cast<unsigned __int128>(hi[i]) << 64) | lo[i];
    std::string text;
    if (s == 0) text = "0";
    while (s > 0) {
      text.insert(text.begin(), static_cast<char>('0' + static_cast<int>(s % 10)));
      s /= 10;
    }
    states.push(Value::string(text));
  }
  out.set("states", std::move(states));
  return out;
}

// OperatorExpressionRequest::Model (bindings/capi/src/lib.rs:791-798): a
// registered model with optional parameter values and the normal action
// (OperatorActionRequest, lib.rs:937-945; transpose, conjugate and adjoint
// actions are not built).
// Matrix, scale, transform and binary expressions build operator algebra
// outside the GPU engine.
// A linear operator expression flattened to (model, parameters, coefficient)
// parts: Model, Scale and Binary add/subtract of OperatorExpressionRequest
// (bindings/capi/src/lib.rs:789-818) with the normal action.
struct ExpressionPart {
  std::shared_ptr<Model> model;
  const Value* parameters;
  C64 coefficient;
  Action action;
};

Action compose(Action a, Action b) {  // actions as (adjoint, conjugate) bits; composition is XOR
  const bool adj = uses_adjoint(a) != uses_adjoint(b), conj = conjugates(a) != conjugates(b);
  if (adj && conj) return Action::kTranspose;
  if (adj) return Action::kAdjoint;
  return conj ? Action::kConjugate : Action::kNormal;
}

// `outer` is the action applied to this subexpression. Adjoints are taken term
// by term, so they conjugate scale coefficients; the conjugating actions are
// applied to the whole result by the caller (conj(c A) keeps c inside).
void flatten_expression(const Value& e, C64 scale, std::vector<ExpressionPart>& parts, Action outer = Action::kNormal) {
  const std::string kind = e.at("kind").as_string();
  if (kind == "model") {
    parts.push_back({registered_model(e.at("handle").as_string()), e.find("parameters"), scale,
                     compose(outer, parse_action(e))});
    return;
  }
  if (kind == "transform") {
    flatten_expression(e.at("operand"), scale, parts, compose(outer, parse_action(e)));
    return;
  }
  if (kind == "scale") {
    const auto& c = e.at("coefficient").items();
    if (c.size() != 2) raise(QMBED_INVALID_OPTIONS, "coefficients are [re, im] pairs");
    C64 coefficient(c[0].as_double(), c[1].as_double());
    if (uses_adjoint(outer)) coefficient = std::conj(coefficient);
    flatten_expression(e.at("operand"), scale * coefficient, parts, outer);
    return;
  }
  if (kind == "binary") {
    const std::string op = e.at("operation").as_string();
    if (op != "add" && op != "subtract")
      raise(QMBED_UNSUPPORTED_BACKEND, "operator products are outside the GPU engine");
    flatten_expression(e.at("left"), scale, parts, outer);
    flatten_expression(e.at("right"), op == "add" ? scale : -scale, parts, outer);
    return;
  }
  raise(QMBED_UNSUPPORTED_BACKEND, "operator expressions of kind `" + kind + "` are outside the GPU engine");
}

bool same_space(const Model& a, const Model& b) {
  const SectorParams& x = a.basis->params();
  const SectorParams& y = b.basis->params();
  return x.sites == y.sites && x.up == y.up && x.has_momentum == y.has_momentum && x.momentum == y.momentum &&
         x.parity == y.parity && x.inversion == y.inversion && a.basis->normalization() == b.basis->normalization() &&
         a.convention.same_sites(b.convention) && a.convention.flipped == b.convention.flipped;
}

// The operator of a linear expression. Adjoints are built from adjoint
// terms; a conjugating action (conjugate, transpose) is returned through
// `conjugate` for the caller to apply as conj(A conj(x)) or to conjugate
// entries, and is refused when the caller cannot (`conjugate` null) or when
// parts disagree on it.
std::shared_ptr<qmbed_operator_s> expression_operator(const Value& e, int storage = kStoragePacked,
                                                      bool* conjugate = nullptr) {
  std::vector<ExpressionPart> parts;
  flatten_expression(e, C64(1.0, 0.0), parts);
  const bool conj = conjugates(parts[0].action);
  for (const ExpressionPart& part : parts)
    if (conjugates(part.action) != conj)
      raise(QMBED_UNSUPPORTED_BACKEND, "sums of conjugated and plain operators are outside the GPU engine");
  if (conj && !conjugate)
    raise(QMBED_UNSUPPORTED_BACKEND, "conjugate and transpose actions are applied or evaluated only");
  if (conjugate) *conjugate = conj;
  if (parts.size() == 1 && parts[0].coefficient == C64(1.0, 0.0))
    return parts[0].model->materialize_action(parts[0].parameters, storage, parts[0].action);
  Model& first = *parts[0].model;
  std::string key = "expression|" + std::to_string(storage);
  std::vector<TermDesc> all;
  for (const ExpressionPart& part : parts) {
    if (!same_space(first, *part.model))
      raise(QMBED_DIMENSION_MISMATCH, "operator expression terms act on different spaces");
    char buffer[160];
    std::snprintf(buffer, sizeof(buffer), "|%llu%s*%.17g,%.17g", static_cast<unsigned long long>(part.model->id),
                  uses_adjoint(part.action) ? "^" : "", part.coefficient.real(), part.coefficient.imag());
    key += buffer;
    std::vector<TermDesc> terms = part.model->resolved_terms(part.parameters, key);
    if (uses_adjoint(part.action)) terms = adjoint_terms(terms);
    for (TermDesc t : terms) {
      for (auto& coupling : t.couplings) coupling.coefficient *= part.coefficient;
      all.push_back(std::move(t));
    }
  }
  OperatorChecks c = first.checks;
  c.hermiticity = false;
  return first.cached(key, all, c, storage);
}

// ExpmActionPlan applied to a host column batch (the apply step of
// ExpmMultiplyParallel, src/solve/mod.rs:252-326), one column at a time.
Value expm_vectors(const LinearOperatorView& view, BlockOps& ops, const ExpmPlan& plan,
                   const std::vector<std::vector<C64>>& vectors) {
  const uint64_t dim = view.dim;
  DeviceBuffer state(std::max<uint64_t>(dim, 1) * 16);
  std::vector<double> host(2 * dim);
  Value out = Value::object();
  out.set("kind", Value::string("vectors"));
  out.set("dimension", Value::integer(static_cast<long long>(vectors.empty() ? dim : vectors[0].size())));
  Value vs = Value::array();
  for (const auto& v : vectors) {
    if (v.size() != dim) raise(QMBED_DIMENSION_MISMATCH, "exponential batch column has the wrong length");
    for (uint64_t i = 0; i < dim; ++i) {
      host[2 * i] = v[i].real();
      host[2 * i + 1] = v[i].imag();
    }
    QMBED_CUDA(cudaMemcpy(state.get(), host.data(), 16 * dim, cudaMemcpyHostToDevice));
    expm_apply(plan, view, state.get(), 64, ops);
    QMBED_CUDA(cudaMemcpy(host.data(), state.get(), 16 * dim, cudaMemcpyDeviceToHost));
    Value r = Value::array();
    for (uint64_t i = 0; i < dim; ++i) r.push(complex_pair(C64(host[2 * i], host[2 * i + 1])));
    vs.push(std::move(r));
  }
  out.set("vectors", std::move(vs));
  return out;
}

Value expm_vectors(qmbed_operator_s& h, const ExpmPlan& plan, const std::vector<std::vector<C64>>& vectors) {
  std::lock_guard<std::mutex> lock(h.mu);
  return expm_vectors(h.view(), h.block_ops(), plan, vectors);
}

// create_expm_action / expm_operator_expression options: ExpmMultiplyParallel
// defaults 55 / eps/2 / 10000 (bindings/capi/src/lib.rs:2111-2121).
ExpmPlan expm_plan_from(const Value& request, qmbed_operator_s& op) {
  const auto& c = request.at("coefficient").items();
  if (c.size() != 2) raise(QMBED_INVALID_OPTIONS, "coefficient is a [re, im] pair");
  const C64 coefficient(c.at(0).as_double(), c.at(1).as_double());
  const size_t max_degree = request.has("max_degree") ? static_cast<size_t>(request.at("max_degree").as_int()) : 55;
  const double tolerance = request.has("tolerance") ? request.at("tolerance").as_double() : 0.5 * 2.220446049250313e-16;
  const size_t substeps = request.has("max_substeps") ? static_cast<size_t>(request.at("max_substeps").as_int()) : 10000;
  return make_expm_plan(*op.op, coefficient, max_degree, tolerance, substeps);
}

// command_eigh (bindings/capi/src/lib.rs:5290-5300) in the command_eigensystem layout.
Value dense_eigh_value(qmbed_operator_s& h, bool want_vectors) {
  std::lock_guard<std::mutex> lock(h.mu);
  const DenseEigensystem r = dense_eigh(h.view(), want_vectors, h.block_ops());
  const uint64_t n = h.op->dim();
  Value out = Value::object();
  out.set("kind", Value::string("eigensystem"));
  out.set("dimension", Value::integer(static_cast<long long>(n)));
  Value vals = Value::array(), res = Value::array();
  for (double v : r.eigenvalues) vals.push(Value::number(v));
  for (double v : r.residuals) res.push(Value::number(v));
  out.set("eigenvalues", std::move(vals));
  out.set("residuals", std::move(res));
  out.set("iterations", Value::integer(n != 0 ? 1 : 0));
  out.set("converged", Value::boolean(true));
  if (want_vectors) {
    std::vector<double> host(2 * r.vectors.size());
    for (size_t i = 0; i < r.vectors.size(); ++i) {
      host[2 * i] = r.vectors[i].real();
      host[2 * i + 1] = r.vectors[i].imag();
    }
    out.set("eigenvectors", vectors_value(host, n, r.eigenvalues.size()));
  }
  return out;
}

// The assembled rows as the reference's operator payload: shape, format and
// (row, column, value) entries in row order.
Value operator_entries(qmbed_operator_s& h, const std::string& format, bool conjugate = false) {
  std::lock_guard<std::mutex> lock(h.mu);
  std::vector<uint64_t> row_ptr;
  std::vector<uint32_t> cols;
  std::vector<C64> values;
  h.op->export_csr(row_ptr, cols, values);
  Value out = Value::object();
  out.set("kind", Value::string("operator"));
  Value shape = Value::array();
  shape.push(Value::integer(static_cast<long long>(h.op->dim())));
  shape.push(Value::integer(static_cast<long long>(h.op->dim())));
  out.set("shape", std::move(shape));
  out.set("format", Value::string(format));
  Value entries = Value::array();
  for (uint64_t r = 0; r + 1 < row_ptr.size(); ++r)
    for (uint64_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
      Value e = Value::object();
      e.set("row", Value::integer(static_cast<long long>(r)));
      e.set("column", Value::integer(static_cast<long long>(cols[p])));
      e.set("value", complex_pair(conjugate ? std::conj(values[p]) : values[p]));
      entries.push(std::move(e));
    }
  out.set("entries", std::move(entries));
  return out;
}

Value command(const Value& request) {
  const std::string operation = request.at("operation").as_string();
  if (operation == "describe_basis") return describe_basis(request);
  if (operation == "create_operator_model") {
    if (request.has("basis")) raise(QMBED_UNSUPPORTED_BACKEND, "basis-embedded operator models are not supported by the GPU engine");
    if (const Value* c = request.find("components"); c && c->is_array() && !c->items().empty())
      raise(QMBED_UNSUPPORTED_BACKEND, "operator models with matrix components are not supported by the GPU engine");
    if (!request.has("static_operator")) raise(QMBED_INVALID_OPTIONS, "an operator model needs a static operator");
    auto model = std::make_shared<MatrixModel>();
    model->matrix = parse_matrix(request.at("static_operator"));
    const uint64_t id = g_next_model.fetch_add(1);
    {
      std::lock_guard<std::mutex> lock(g_registry_mu);
      g_matrix_models[id] = model;
    }
    Value out = Value::object();
    out.set("kind", Value::string("model"));
    out.set("handle", Value::string(std::to_string(id)));
    out.set("dimension", Value::integer(static_cast<long long>(model->matrix->dim())));
    return out;
  }
  if (operation == "create_expm_action" || operation == "apply_model" || operation == "eigsh_model") {
    if (auto mm = matrix_model(request.at("handle").as_string())) {
      if (request.has("parameters") && request.at("parameters").is_object() && !request.at("parameters").members().empty())
        raise(QMBED_INVALID_OPTIONS, "this operator model has no parameters");
      std::lock_guard<std::mutex> lock(mm->mu);
      if (operation == "apply_model") {
        if (request.has("action") && request.at("action").as_string() != "normal")
          raise(QMBED_UNSUPPORTED_BACKEND, "only the normal action is supported by the GPU engine");
        return vectors_result(apply_columns(mm->view(), mm->block_ops(), parse_vectors(request.at("vectors")),
                                            "vector length does not match the model dimension"),
                              mm->matrix->dim());
      }
      if (operation == "eigsh_model") return solve_view(mm->view(), mm->block_ops(), parse_solver(request.at("solver")), true);
      auto entry = std::make_shared<ExpmEntry>();
      entry->matrix = mm;
      const auto& c = request.at("coefficient").items();
      if (c.size() != 2) raise(QMBED_INVALID_OPTIONS, "coefficient is a [re, im] pair");
      const size_t max_degree = request.has("max_degree") ? static_cast<size_t>(request.at("max_degree").as_int()) : 55;
      const double tolerance = request.has("tolerance") ? request.at("tolerance").as_double() : 0.5 * 2.220446049250313e-16;
      const size_t substeps = request.has("max_substeps") ? static_cast<size_t>(request.at("max_substeps").as_int()) : 10000;
      entry->plan = make_expm_plan(mm->matrix->dim(), mm->matrix->shift(), mm->matrix->one_norm(),
                                   C64(c[0].as_double(), c[1].as_double()), max_degree, tolerance, substeps);
      const uint64_t id = g_next_expm.fetch_add(1);
      {
        std::lock_guard<std::mutex> registry(g_registry_mu);
        g_expm[id] = entry;
      }
      Value out = Value::object();
      out.set("kind", Value::string("expm_plan"));
      out.set("handle", Value::string(std::to_string(id)));
      out.set("dimension", Value::integer(static_cast<long long>(mm->matrix->dim())));
      return out;
    }
  }
  if (operation == "eigsh") {
    auto model = build_model(request);
    auto op = model->materialize(nullptr, parse_storage(request), true);
    return solve(*op, parse_solver(request.at("solver")), true);
  }
  if (operation == "materialize") {
    auto model = build_model(request);
    auto op = model->materialize(nullptr, kStoragePacked, model->checks.hermiticity);
    return operator_entries(*op, request.has("format") ? request.at("format").as_string() : "csc");
  }
  if (operation == "materialize_model") {
    // MaterializeModel -> command_operator (bindings/capi/src/lib.rs:5652-5659)
    auto model = registered_model(request.at("handle").as_string());
    auto op = model->materialize(request.find("parameters"), kStoragePacked, false);
    return operator_entries(*op, request.has("format") ? request.at("format").as_string() : "csc");
  }
  if (operation == "materialize_component_model") {
    // MaterializeComponentModel -> component_operator (bindings/capi/src/lib.rs:5797-5805,
    // src/interop.rs:185-190): one named component with coefficient 1
    auto model = registered_model(request.at("handle").as_string());
    const std::string name = request.at("name").as_string();
    if (model->components.empty()) raise(QMBED_INVALID_OPTIONS, "fixed operator model has no component \"" + name + "\"");
    const Component* found = nullptr;
    for (const Component& c : model->components)
      if (c.name == name) found = &c;
    if (!found) raise(QMBED_INVALID_OPTIONS, "unknown operator component \"" + name + "\"");
    OperatorChecks checks = model->checks;
    checks.hermiticity = false;
    auto op = model->cached("component|" + name, found->terms, checks, kStoragePacked);
    return operator_entries(*op, request.has("format") ? request.at("format").as_string() : "csc");
  }
  if (operation == "evaluate_operator_expression") {
    // EvaluateOperatorExpression -> command_operator_value (bindings/capi/src/lib.rs:5660-5663)
    bool conj = false;
    auto op = expression_operator(request.at("expression"), kStoragePacked, &conj);
    return operator_entries(*op, request.has("format") ? request.at("format").as_string() : "csc", conj);
  }
  if (operation == "create_model") {
    auto model = build_model(request);
    const uint64_t id = g_next_model.fetch_add(1);
    model->id = id;
    {
      std::lock_guard<std::mutex> lock(g_registry_mu);
      g_models[id] = model;
    }
    Value out = Value::object();
    out.set("kind", Value::string("model"));
    out.set("handle", Value::string(std::to_string(id)));
    out.set("dimension", Value::integer(static_cast<long long>(model->basis->dim())));
    return out;
  }
  if (operation == "describe_model") {
    auto model = registered_model(request.at("handle").as_string());
    Value out = Value::object();
    out.set("kind", Value::string("model"));
    out.set("handle", Value::string(request.at("handle").as_string()));
    out.set("dimension", Value::integer(static_cast<long long>(model->basis->dim())));
    return out;
  }
  if (operation == "eigsh_model") {
    auto model = registered_model(request.at("handle").as_string());
    auto op = model->materialize(request.find("parameters"), parse_storage(request), true);
    return solve(*op, parse_solver(request.at("solver")), true);
  }
  if (operation == "apply_model") {
    auto model = registered_model(request.at("handle").as_string());
    // OperatorActionRequest (bindings/capi/src/lib.rs:937-945): "normal" is the default
    const Action action = parse_action(request);
    auto op = model->materialize_action(request.find("parameters"), kStoragePacked, action);
    return apply_with_action(*op, parse_vectors(request.at("vectors")), conjugates(action));
  }
  if (operation == "matrix_elements_model") return matrix_elements(*registered_model(request.at("handle").as_string()), request);
  if (operation == "measure_model") return measure(*registered_model(request.at("handle").as_string()), request);
  if (operation == "create_expm_action") {
    auto model = registered_model(request.at("handle").as_string());
    auto op = model->materialize(request.find("parameters"), kStoragePacked, false);
    auto entry = std::make_shared<ExpmEntry>();
    entry->op = op;
    entry->plan = expm_plan_from(request, *op);
    const uint64_t id = g_next_expm.fetch_add(1);
    {
      std::lock_guard<std::mutex> lock(g_registry_mu);
      g_expm[id] = entry;
    }
    Value out = Value::object();
    out.set("kind", Value::string("expm_plan"));
    out.set("handle", Value::string(std::to_string(id)));
    out.set("dimension", Value::integer(static_cast<long long>(op->op->dim())));
    return out;
  }
  if (operation == "apply_expm_action") {
    auto entry = registered_expm(request.at("expm_handle").as_string());
    if (entry->matrix) {
      std::lock_guard<std::mutex> lock(entry->matrix->mu);
      return expm_vectors(entry->matrix->view(), entry->matrix->block_ops(), entry->plan,
                          parse_vectors(request.at("vectors")));
    }
    return expm_vectors(*entry->op, entry->plan, parse_vectors(request.at("vectors")));
  }
  if (operation == "eigh_model") {
    // command_eigh (bindings/capi/src/lib.rs:5290-5300)
    auto model = registered_model(request.at("handle").as_string());
    auto op = model->materialize(request.find("parameters"), kStoragePacked, false);
    return dense_eigh_value(*op, request.has("eigenvectors") && request.at("eigenvectors").as_bool());
  }
  if (operation == "eigh_operator_expression") {
    auto op = expression_operator(request.at("expression"));
    return dense_eigh_value(*op, request.has("eigenvectors") && request.at("eigenvectors").as_bool());
  }
  if (operation == "eigsh_operator_expression") {
    // command_eigsh_operator_expression (bindings/capi/src/lib.rs:4172-4190)
    auto op = expression_operator(request.at("expression"), parse_storage(request));
    return solve(*op, parse_solver(request.at("solver")), true);
  }
  if (operation == "apply_operator_expression") {
    // command_apply_operator_expression (bindings/capi/src/lib.rs:4078-4105)
    bool conj = false;
    auto op = expression_operator(request.at("expression"), kStoragePacked, &conj);
    const auto vectors = parse_vectors(request.at("vectors"));
    bool ok = !vectors.empty();
    for (const auto& v : vectors) ok = ok && v.size() == op->op->dim();
    if (!ok) raise(QMBED_DIMENSION_MISMATCH, "operator expression inputs must be a nonempty batch matching its columns");
    return apply_with_action(*op, vectors, conj);
  }
  if (operation == "expm_operator_expression") {
    // command_expm_operator_expression (bindings/capi/src/lib.rs:4135-4170)
    auto op = expression_operator(request.at("expression"));
    const ExpmPlan plan = expm_plan_from(request, *op);
    const auto vectors = parse_vectors(request.at("vectors"));
    if (vectors.empty()) raise(QMBED_INVALID_OPTIONS, "operator exponential requires a nonempty vector batch");
    return expm_vectors(*op, plan, vectors);
  }
  if (operation == "evolve_model") {
    // command_evolve_model (bindings/capi/src/lib.rs:4673-4694), EvolutionRequest
    // defaults 64 / 1e-10 / 10000 (lib.rs:431-441, 596-606)
    auto model = registered_model(request.at("handle").as_string());
    const Value& ev = request.at("evolution");
    if (ev.has("imaginary_time") && ev.at("imaginary_time").as_bool())
      raise(QMBED_INVALID_OPTIONS, "static imaginary-time evolution is not exposed by this command yet");
    EvolutionOptions o;
    for (const Value& t : ev.at("times").items()) o.times.push_back(t.as_double());
    o.krylov_dimension = ev.has("krylov_dimension") ? static_cast<size_t>(ev.at("krylov_dimension").as_int()) : 64;
    o.tolerance = ev.has("tolerance") ? ev.at("tolerance").as_double() : 1.0e-10;
    o.max_substeps = ev.has("max_substeps") ? static_cast<size_t>(ev.at("max_substeps").as_int()) : 10000;
    auto vectors = parse_vectors(request.at("vectors"));
    if (vectors.empty()) raise(QMBED_INVALID_OPTIONS, "a state batch must contain at least one column");
    auto op = model->materialize(request.find("parameters"), kStoragePacked, true);
    qmbed_operator_s& h = *op;
    std::lock_guard<std::mutex> lock(h.mu);
    const uint64_t dim = h.op->dim();
    std::vector<std::vector<double>> per_column;
    for (const auto& v : vectors) {
      if (v.size() != dim) raise(QMBED_DIMENSION_MISMATCH, "evolution operator and initial state do not match");
      std::vector<double> host(2 * dim), states(2 * dim * o.times.size());
      for (uint64_t i = 0; i < dim; ++i) {
        host[2 * i] = v[i].real();
        host[2 * i + 1] = v[i].imag();
      }
      EvolutionDiagnostics d;
      evolve(h.view(), host.data(), o, states.data(), d, h.block_ops());
      per_column.push_back(std::move(states));
    }
    Value out = Value::object();
    out.set("kind", Value::string("trajectory"));
    out.set("dimension", Value::integer(static_cast<long long>(dim)));
    Value times = Value::array();
    for (double t : o.times) times.push(Value::number(t));
    out.set("times", std::move(times));
    Value states = Value::array();
    for (size_t t = 0; t < o.times.size(); ++t) {
      Value columns = Value::array();
      for (const auto& col : per_column) {
        Value r = Value::array();
        for (uint64_t i = 0; i < dim; ++i) r.push(complex_pair(C64(col[2 * (t * dim + i)], col[2 * (t * dim + i) + 1])));
        columns.push(std::move(r));
      }
      states.push(std::move(columns));
    }
    out.set("states", std::move(states));
    return out;
  }
  if (operation == "apply_terms_between_models") {
    // registered_cross_sector_action (bindings/capi/src/lib.rs:4871-4915) for
    // two spin-sector models: apply_sector_shift of the request's terms
    auto source = registered_model(request.at("source_handle").as_string());
    auto target = registered_model(request.at("target_handle").as_string());
    if (!source->convention.same_sites(target->convention))
      raise(QMBED_INVALID_OPTIONS, "models must use the same site permutation for cross-basis operations");
    if (source->convention.flipped != target->convention.flipped)
      raise(QMBED_UNSUPPORTED_BACKEND, "cross-sector actions between reversed and ordinary bases are not supported by "
                                       "the GPU engine");
    const auto terms = source->convention.prepare(parse_terms(request.at("terms")));
    const auto vectors = parse_vectors(request.at("vectors"));
    OperatorChecks checks;
    checks.hermiticity = false;
    checks.particle_conservation = false;
    if (source->basis->sites() != target->basis->sites() ||
        source->basis->normalization() != target->basis->normalization())
      raise(QMBED_INVALID_OPTIONS, "source and target models use different site conventions");
    SpinOperator shift(source->basis, terms, checks, kStorageMatrixFree);
    const uint64_t ns = source->basis->dim(), nt = target->basis->dim();
    cudaStream_t stream;
    QMBED_CUDA(cudaSetDevice(source->basis->device()));
    QMBED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    std::vector<double> host;
    try {
      DeviceBuffer dx(std::max<uint64_t>(ns, 1) * 16), dy(std::max<uint64_t>(nt, 1) * 16);
      std::vector<double> in(2 * ns), out(2 * nt);
      for (const auto& v : vectors) {
        if (v.size() != ns)
          raise(QMBED_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
        for (uint64_t i = 0; i < ns; ++i) {
          in[2 * i] = v[i].real();
          in[2 * i + 1] = v[i].imag();
        }
        QMBED_CUDA(cudaMemcpyAsync(dx.get(), in.data(), ns * 16, cudaMemcpyHostToDevice, stream));
        shift.apply_shift(*target->basis, dx.as<double>(), dy.as<double>(), stream);
        QMBED_CUDA(cudaMemcpyAsync(out.data(), dy.get(), nt * 16, cudaMemcpyDeviceToHost, stream));
        QMBED_CUDA(cudaStreamSynchronize(stream));
        host.insert(host.end(), out.begin(), out.end());
      }
    } catch (...) {
      cudaStreamDestroy(stream);
      throw;
    }
    cudaStreamDestroy(stream);
    Value out = Value::object();
    out.set("kind", Value::string("vectors"));
    out.set("dimension", Value::integer(static_cast<long long>(nt)));
    out.set("vectors", vectors_value(host, nt, vectors.size()));
    return out;
  }
  if (operation == "lanczos_operator") {
    // command_lanczos_operator (bindings/capi/src/lib.rs:4046-4075); tolerance
    // default 1e-13 (default_lanczos_tolerance, lib.rs:2107-2109)
    auto op = expression_operator(request.at("expression"));
    const long long krylov = request.at("krylov_dimension").as_int();
    if (krylov < 0) raise(QMBED_INVALID_OPTIONS, "krylov_dimension must be a nonnegative integer");
    const double tolerance = request.has("tolerance") ? request.at("tolerance").as_double() : 1.0e-13;
    const auto initial = parse_vector(request.at("initial"));
    auto entry = std::make_shared<qmbed_lanczos_s>();
    {
      std::lock_guard<std::mutex> lock(op->mu);
      const uint64_t dim = op->op->dim();
      validate_lanczos(static_cast<size_t>(krylov), tolerance);
      if (initial.size() != dim) raise(QMBED_DIMENSION_MISMATCH, "Lanczos operator and initial vector do not match");
      std::vector<double> host(2 * dim);
      for (uint64_t i = 0; i < dim; ++i) {
        host[2 * i] = initial[i].real();
        host[2 * i + 1] = initial[i].imag();
      }
      lanczos_ritz(op->view(), host.data(), static_cast<size_t>(krylov), tolerance, entry->d, op->block_ops());
    }
    const uint64_t id = g_next_lanczos.fetch_add(1);
    {
      std::lock_guard<std::mutex> lock(g_registry_mu);
      g_lanczos[id] = entry;
    }
    const LanczosDecomposition& d = entry->d;
    Value out = Value::object();
    out.set("kind", Value::string("lanczos"));
    out.set("handle", Value::string("lanczos:" + std::to_string(id)));
    out.set("dimension", Value::integer(static_cast<long long>(initial.size())));
    out.set("krylov_dimension", Value::integer(d.size));
    out.set("initial_norm", Value::number(d.initial_norm));
    Value values = Value::array(), vectors = Value::array();
    for (int c = 0; c < d.size; ++c) {
      values.push(Value::number(d.eigenvalues[c]));
      Value v = Value::array();
      for (int r = 0; r < d.size; ++r) v.push(Value::number(d.vec(r, c)));
      vectors.push(std::move(v));
    }
    out.set("eigenvalues", std::move(values));
    out.set("eigenvectors", std::move(vectors));
    return out;
  }
  if (operation == "lanczos_combine" || operation == "lanczos_exponential") {
    // command_lanczos_combine / command_lanczos_exponential (bindings/capi/src/lib.rs:4192-4212)
    auto entry = registered_lanczos(request.at("lanczos_handle").as_string());
    std::lock_guard<std::mutex> lock(entry->mu);
    std::vector<C64> c;
    if (operation == "lanczos_combine") {
      c = parse_vector(request.at("coefficients"));
    } else {
      const auto& pair = request.at("coefficient").items();
      if (pair.size() != 2) raise(QMBED_INVALID_OPTIONS, "coefficient is a [re, im] pair");
      c = exponential_coefficients(entry->d, C64(pair[0].as_double(), pair[1].as_double()));
    }
    std::vector<double> host(2 * entry->d.n);
    lanczos_vector_out(*entry, c, host.data());
    Value out = Value::object();
    out.set("kind", Value::string("vectors"));
    out.set("dimension", Value::integer(static_cast<long long>(entry->d.n)));
    out.set("vectors", vectors_value(host, entry->d.n, 1));
    return out;
  }
  if (operation == "lanczos_thermal") {
    // command_lanczos_thermal (bindings/capi/src/lib.rs:4214-4291): the
    // eigenvector matrix arrives row-major; observables carry either a model
    // expression (projected on the GPU through the handle's basis) or their
    // projected matrix elements.
    const std::string method_name = request.at("method").as_string();
    if (method_name != "ftlm" && method_name != "ltlm") raise(QMBED_INVALID_OPTIONS, "method must be `ftlm` or `ltlm`");
    const bool ltlm = method_name == "ltlm";
    std::vector<double> eigenvalues;
    for (const Value& v : request.at("eigenvalues").items()) eigenvalues.push_back(v.as_double());
    const size_t m = eigenvalues.size();
    const auto& rows = request.at("eigenvectors").items();
    if (rows.size() != m) raise(QMBED_DIMENSION_MISMATCH, "Lanczos Ritz eigenvectors must be a square row-major matrix");
    std::vector<std::vector<double>> columns(m, std::vector<double>(m));
    for (size_t r = 0; r < m; ++r) {
      const auto& row = rows[r].items();
      if (row.size() != m) raise(QMBED_DIMENSION_MISMATCH, "Lanczos Ritz eigenvectors must be a square row-major matrix");
      for (size_t c = 0; c < m; ++c) columns[c][r] = row[c].as_double();
    }
    std::vector<double> betas;
    for (const Value& v : request.at("inverse_temperatures").items()) betas.push_back(v.as_double());
    std::vector<std::string> names;
    std::vector<std::vector<C64>> projected;
    std::vector<std::pair<std::string, std::shared_ptr<qmbed_operator_s>>> native;
    for (const Value& o : request.at("observables").items()) {
      const bool has_expression = o.has("expression") && !o.at("expression").is_null();
      const bool has_elements = o.has("matrix_elements") && !o.at("matrix_elements").items().empty();
      if (has_expression == has_elements)
        raise(QMBED_INVALID_OPTIONS, "each thermal observable needs exactly one expression or projected matrix");
      if (has_expression) {
        native.emplace_back(o.at("name").as_string(), expression_operator(o.at("expression")));
      } else {
        names.push_back(o.at("name").as_string());
        projected.push_back(parse_vector(o.at("matrix_elements")));
      }
    }
    if (!native.empty()) {
      if (!request.has("lanczos_handle") || request.at("lanczos_handle").is_null())
        raise(QMBED_INVALID_OPTIONS, "native thermal observables require a Lanczos handle");
      auto entry = registered_lanczos(request.at("lanczos_handle").as_string());
      std::lock_guard<std::mutex> lock(entry->mu);
      if (static_cast<size_t>(entry->d.size) != m)
        raise(QMBED_DIMENSION_MISMATCH, "Lanczos handle and supplied Ritz eigensystem dimensions differ");
      for (auto& [name, op] : native) {
        std::lock_guard<std::mutex> olock(op->mu);
        names.push_back(name);
        projected.push_back(project_observable(entry->d, op->view(), ltlm, op->block_ops()));
      }
    }
    for (size_t i = 0; i < names.size(); ++i) {
      bool unique = !names[i].empty();
      for (size_t j = 0; j < i; ++j) unique = unique && names[j] != names[i];
      if (!unique) raise(QMBED_DIMENSION_MISMATCH, "thermal observables require unique names and matching finite projections");
    }
    std::vector<std::vector<C64>> values;
    std::vector<double> identity;
    thermal_contraction(ltlm, eigenvalues, columns, projected, betas, values, identity);
    Value out = Value::object();
    out.set("kind", Value::string("thermal_lanczos"));
    Value vals = Value::object();
    for (size_t o = 0; o < names.size(); ++o) {
      Value series = Value::array();
      for (const C64& v : values[o]) series.push(complex_pair(v));
      vals.set(names[o], std::move(series));
    }
    out.set("values", std::move(vals));
    Value id = Value::array();
    for (double v : identity) id.push(Value::number(v));
    out.set("identity", std::move(id));
    return out;
  }
  if (operation == "export_lanczos_basis") {
    // command_export_lanczos_basis (bindings/capi/src/lib.rs:4293-4310)
    auto entry = registered_lanczos(request.at("lanczos_handle").as_string());
    std::lock_guard<std::mutex> lock(entry->mu);
    QMBED_CUDA(cudaSetDevice(entry->d.device));
    std::vector<double> host;
    for (int j = 0; j < entry->d.size; ++j) {
      const std::vector<double> col = lanczos_column_host(entry->d, j);
      host.insert(host.end(), col.begin(), col.end());
    }
    Value out = Value::object();
    out.set("kind", Value::string("lanczos_basis"));
    out.set("dimension", Value::integer(static_cast<long long>(entry->d.n)));
    out.set("vectors", vectors_value(host, entry->d.n, static_cast<size_t>(entry->d.size)));
    return out;
  }
  if (operation == "release_lanczos") {
    // release_lanczos (bindings/capi/src/lib.rs:1874-1886)
    const std::string text = request.at("lanczos_handle").as_string();
    const uint64_t id = parse_lanczos_handle(text);
    std::shared_ptr<qmbed_lanczos_s> released;
    {
      std::lock_guard<std::mutex> lock(g_registry_mu);
      auto it = g_lanczos.find(id);
      if (it == g_lanczos.end()) raise(QMBED_INVALID_OPTIONS, "Lanczos handle " + text + " is not registered");
      released = std::move(it->second);
      g_lanczos.erase(it);
    }
    Value out = Value::object();
    out.set("kind", Value::string("released"));
    out.set("handle", Value::string("lanczos:" + std::to_string(id)));
    return out;
  }
  if (operation == "release_model") {
    const std::string text = request.at("handle").as_string();
    const uint64_t id = parse_handle(text, "model");
    std::lock_guard<std::mutex> lock(g_registry_mu);
    if (!g_models.erase(id) && !g_matrix_models.erase(id))
      raise(QMBED_INVALID_OPTIONS, "model handle " + text + " is not registered");
    Value out = Value::object();
    out.set("kind", Value::string("released"));
    out.set("handle", Value::string(text));
    return out;
  }
  if (operation == "release_expm_action") {
    const std::string text = request.at("expm_handle").as_string();
    const uint64_t id = parse_handle(text, "exponential-action");
    std::lock_guard<std::mutex> lock(g_registry_mu);
    if (!g_expm.erase(id)) raise(QMBED_INVALID_OPTIONS, "exponential-action handle " + text + " is not registered");
    Value out = Value::object();
    out.set("kind", Value::string("released"));
    out.set("handle", Value::string(text));
    return out;
  }
  raise(QMBED_UNSUPPORTED_BACKEND, "operation `" + operation + "` is outside the GPU engine");
}

std::string respond_with(const char* request, const std::string& invalid,
                         const std::function<Value(const Value&)>& handler) {
  if (!request) return R"({"status":"error","error":"request pointer is null"})";
  CallerDevice restore;
  Value response = Value::object();
  try {
    Value parsed;
    try {
      parsed = json::parse(request);
    } catch (const json::ParseError& e) {
      raise(QMBED_INVALID_OPTIONS, invalid + e.what());
    }
    Value result;
    try {
      result = handler(parsed);
    } catch (const json::ParseError& e) {
      raise(QMBED_INVALID_OPTIONS, invalid + e.what());
    }
    response.set("status", Value::string("ok"));
    response.set("result", std::move(result));
  } catch (const Error& e) {
    response = Value::object();
    response.set("status", Value::string("error"));
    response.set("error", Value::string(e.what()));
  } catch (const std::exception& e) {
    response = Value::object();
    response.set("status", Value::string("error"));
    response.set("error", Value::string(std::string("internal state error: ") + e.what()));
  }
  return response.dump();
}

std::string respond(const char* request, bool command_api) {
  return respond_with(request, command_api ? "invalid binding command: " : "invalid binding request: ",
                      [command_api](const Value& r) { return command_api ? command(r) : run_request(r); });
}

// QmbedComplex64 and the drive callback of qmbed_evolve_model_with_drive_json
// (bindings/capi/src/lib.rs:452-470): fill `count` coefficients at `time`,
// return 0 on success.
struct DriveComplex {
  double real, imaginary;
};
using DriveCallbackFn = int (*)(void*, double, DriveComplex*, size_t);

std::string debug_names(const std::vector<std::string>& names) {
  std::string out = "[";
  for (size_t i = 0; i < names.size(); ++i) out += (i ? ", \"" : "\"") + names[i] + "\"";
  return out + "]";
}

Value drive_evolution(const Value& request, void* callback, void* context) {
  auto model = registered_model(request.at("handle").as_string());
  std::vector<std::string> names, expected;
  for (const Value& v : request.at("component_names").items()) names.push_back(v.as_string());
  for (const Component& c : model->components) expected.push_back(c.name);
  if (names != expected)
    raise(QMBED_INVALID_OPTIONS, "drive component order mismatch: expected " + debug_names(expected) + ", received " +
                                     debug_names(names));
  if (expected.empty()) raise(QMBED_INVALID_OPTIONS, "time-dependent evolution requires at least one operator component");
  const Value& ev = request.at("evolution");
  EvolutionOptions o;
  for (const Value& t : ev.at("times").items()) o.times.push_back(t.as_double());
  o.krylov_dimension = ev.has("krylov_dimension") ? static_cast<size_t>(ev.at("krylov_dimension").as_int()) : 64;
  o.tolerance = ev.has("tolerance") ? ev.at("tolerance").as_double() : 1.0e-10;
  o.max_substeps = ev.has("max_substeps") ? static_cast<size_t>(ev.at("max_substeps").as_int()) : 10000;
  const bool imaginary = ev.has("imaginary_time") && ev.at("imaginary_time").as_bool();
  const double initial_time = request.at("initial_time").as_double();
  const auto vectors = parse_vectors(request.at("vectors"));
  if (vectors.empty()) raise(QMBED_INVALID_OPTIONS, "a state batch must contain at least one column");

  OperatorChecks checks = model->checks;
  checks.hermiticity = false;
  std::vector<std::shared_ptr<qmbed_operator_s>> parts;
  parts.push_back(model->terms.empty() ? nullptr : model->cached("static", model->terms, checks, kStoragePacked));
  for (const Component& c : model->components)
    parts.push_back(model->cached("component|" + c.name, c.terms, checks, kStoragePacked));
  std::vector<std::unique_lock<std::mutex>> locks;
  for (auto& part : parts)
    if (part) locks.emplace_back(part->mu);
  qmbed_operator_s& first = parts[0] ? *parts[0] : *parts[1];
  BlockOps& ops = first.block_ops();
  const cudaStream_t stream = ops.stream();
  const uint64_t dim = first.op->dim();

  TimeDependentOperator td;
  td.dim = dim;
  for (auto& part : parts) {
    if (!part) {  // no static terms: the zero operator
      td.parts.push_back(LinearOperatorView{dim, true, [stream, dim](int, bool cplx, const void*, void* y) {
                                              QMBED_CUDA(cudaMemsetAsync(y, 0, dim * (cplx ? 16 : 8), stream));
                                            }});
      continue;
    }
    SpinOperator* raw = part->op.get();
    td.parts.push_back(LinearOperatorView{dim, raw->is_real(), [raw, stream](int prec, bool cplx, const void* x, void* y) {
                                            raw->apply(prec, cplx, x, y, stream);
                                          }});
  }
  auto fn = reinterpret_cast<DriveCallbackFn>(callback);
  td.coefficients = [fn, context](double t, std::vector<C64>& c) {
    std::vector<DriveComplex> buffer(c.size(), DriveComplex{std::nan(""), std::nan("")});
    const int status = fn(context, t, buffer.data(), buffer.size());
    if (status != 0) {
      char text[64];
      std::snprintf(text, sizeof(text), "%.17g", t);
      raise(QMBED_INVALID_OPTIONS, "drive callback returned status " + std::to_string(status) + " at time " + text);
    }
    for (size_t i = 0; i < c.size(); ++i) c[i] = C64(buffer[i].real, buffer[i].imaginary);
  };
  td.scale = imaginary ? C64(0.0, -1.0) : C64(1.0, 0.0);

  std::vector<std::vector<double>> per_column;
  for (const auto& v : vectors) {
    if (v.size() != dim) raise(QMBED_DIMENSION_MISMATCH, "time-dependent operator and initial state do not match");
    std::vector<double> host(2 * dim), states(2 * dim * o.times.size());
    for (uint64_t i = 0; i < dim; ++i) {
      host[2 * i] = v[i].real();
      host[2 * i + 1] = v[i].imag();
    }
    evolve_time_dependent(td, host.data(), initial_time, o, states.data(), ops);
    per_column.push_back(std::move(states));
  }
  Value out = Value::object();
  out.set("kind", Value::string("trajectory"));
  out.set("dimension", Value::integer(static_cast<long long>(dim)));
  Value times = Value::array();
  for (double t : o.times) times.push(Value::number(t));
  out.set("times", std::move(times));
  Value states = Value::array();
  for (size_t t = 0; t < o.times.size(); ++t) {
    Value columns = Value::array();
    for (const auto& col : per_column) {
      Value r = Value::array();
      for (uint64_t i = 0; i < dim; ++i) r.push(complex_pair(C64(col[2 * (t * dim + i)], col[2 * (t * dim + i) + 1])));
      columns.push(std::move(r));
    }
    states.push(std::move(columns));
  }
  out.set("states", std::move(states));
  return out;
}

template <typename F>
char* json_call(const char* request, F handler) {
  return to_c_string(respond_with(request, "invalid drive evolution request: ", handler));
}

}  // namespace

namespace qmbed {

// Status/last-error wrapper and handle access for entry points defined in
// other translation units.
int noalloc_guarded(const std::function<void()>& body) { return guarded(body); }

const SpinOperator& operator_of(qmbed_operator_s* op) {
  if (!op || !op->op) raise(QMBED_INVALID_OPTIONS, "operator handle is null");
  return *op->op;
}

}  // namespace qmbed

extern "C" {

const char* qmbed_gpu_last_error(void) { return g_last_error.c_str(); }

int qmbed_gpu_device_count(int* count) {
  return guarded([&] { QMBED_CUDA(cudaGetDeviceCount(count)); });
}

int qmbed_gpu_launch_count(uint64_t* count) {
  return guarded([&] { *count = g_kernel_launches.load(std::memory_order_relaxed); });
}

int qmbed_gpu_spin_basis_create(int device, int sites, int up, int has_momentum, int momentum, int parity,
                                int normalization, qmbed_basis* out) {
  return guarded([&] {
    SpinBasisDesc d{sites, up, has_momentum, momentum, parity, normalization};
    auto h = new qmbed_basis_s;
    try {
      h->basis = std::make_shared<SpinBasis>(d, device);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int qmbed_gpu_basis_destroy(qmbed_basis basis) {
  return guarded([&] { delete basis; });
}

int qmbed_gpu_basis_dimension(qmbed_basis basis, uint64_t* dimension) {
  return guarded([&] { *dimension = basis->basis->dim(); });
}

int qmbed_gpu_basis_states(qmbed_basis basis, uint64_t offset, uint64_t count, uint64_t* lo, uint64_t* hi,
                           uint16_t* orbit) {
  return guarded([&] { basis->basis->copy_states(offset, count, lo, hi, orbit); });
}

int qmbed_gpu_basis_images(qmbed_basis basis, const uint64_t* lo, const uint64_t* hi, uint64_t n, int64_t* index,
                           double* phase, uint16_t* orbit) {
  return guarded([&] { basis->basis->images(lo, hi, n, index, phase, orbit); });
}

int qmbed_gpu_basis_table_images(qmbed_basis basis, const uint64_t* lo, uint64_t n, int64_t* index, double* phase,
                                 uint16_t* orbit) {
  return guarded([&] {
    if (basis->basis->words() != 1 || !basis->basis->symmetric())
      raise(QMBED_UNSUPPORTED_BACKEND, "image tables serve symmetry sectors of at most 64 sites");
    basis->basis->table_images(lo, n, index, phase, orbit);
  });
}

int qmbed_gpu_basis_build_seconds(qmbed_basis basis, double* seconds) {
  return guarded([&] { *seconds = basis->basis->build_seconds(); });
}

int qmbed_gpu_operator_create(qmbed_basis basis, int n_terms, const int* arity, const char* symbols,
                              const int* n_couplings, const double* coefficients, const int* sites,
                              int check_hermitian, int check_particles, int storage, qmbed_operator* out) {
  return guarded([&] {
    auto terms = decode_terms(n_terms, arity, symbols, n_couplings, coefficients, sites);
    OperatorChecks checks;
    checks.hermiticity = check_hermitian != 0;
    checks.particle_conservation = check_particles != 0;
    auto h = new qmbed_operator_s;
    try {
      if (storage < 0 || storage > 2) raise(QMBED_INVALID_OPTIONS, "storage must be matrix_free, packed or explicit");
      h->op = std::make_shared<SpinOperator>(basis->basis, terms, checks, storage);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int qmbed_gpu_operator_destroy(qmbed_operator op) {
  return guarded([&] { delete op; });
}

int qmbed_gpu_operator_info(qmbed_operator op, uint64_t* dimension, int* is_real, int* storage, uint64_t* nnz_offdiag,
                            int* value_codes, double* assembly_seconds) {
  return guarded([&] {
    if (dimension) *dimension = op->op->dim();
    if (is_real) *is_real = op->op->is_real() ? 1 : 0;
    if (storage) *storage = op->op->storage();
    if (nnz_offdiag) *nnz_offdiag = op->op->nnz_offdiag();
    if (value_codes) *value_codes = op->op->value_codes();
    if (assembly_seconds) *assembly_seconds = op->op->assembly_seconds();
  });
}

int qmbed_gpu_operator_apply_device(qmbed_operator op, int precision, int complex_vectors, const void* x, void* y,
                                    void* stream, int force_matrix_free) {
  return guarded([&] {
    if (precision != 64 && precision != 32) raise(QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
    op->op->apply(precision, complex_vectors != 0, x, y, static_cast<cudaStream_t>(stream), force_matrix_free != 0);
  });
}

int qmbed_gpu_operator_apply_rows_device(qmbed_operator op, int precision, uint64_t row0, uint64_t rows,
                                         const void* x, void* y, void* stream) {
  return guarded([&] {
    if (precision != 64 && precision != 32) raise(QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
    if (!x || !y || x == y) raise(QMBED_INVALID_OPTIONS, "row slabs need distinct input and output vectors");
    op->op->apply_rows(precision, row0, rows, x, y, static_cast<cudaStream_t>(stream));
  });
}

int qmbed_gpu_operator_apply_block_device(qmbed_operator op, int precision, int nb, const void* z, const void* p,
                                          void* out, double alpha, double beta, double gamma, void* stream) {
  return guarded([&] {
    if (precision != 64 && precision != 32) raise(QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
    if (nb != 8 && nb != 16) raise(QMBED_INVALID_OPTIONS, "block width must be 8 or 16");
    if (!z || !out || z == out) raise(QMBED_INVALID_OPTIONS, "block action needs distinct input and output blocks");
    op->op->apply_block(precision, nb, z, p, out, alpha, beta, gamma, static_cast<cudaStream_t>(stream));
  });
}

int qmbed_gpu_operator_apply_host(qmbed_operator op, int complex_vectors, const double* x, double* y,
                                  int force_matrix_free) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(op->mu);
    const uint64_t n = op->op->dim();
    const size_t bytes = std::max<uint64_t>(n, 1) * 8 * (complex_vectors ? 2 : 1);
    BlockOps& ops = op->block_ops();
    DeviceBuffer dx(bytes), dy(bytes);
    QMBED_CUDA(cudaMemcpyAsync(dx.get(), x, n * 8 * (complex_vectors ? 2 : 1), cudaMemcpyHostToDevice, ops.stream()));
    op->op->apply(64, complex_vectors != 0, dx.get(), dy.get(), ops.stream(), force_matrix_free != 0);
    QMBED_CUDA(cudaMemcpyAsync(y, dy.get(), n * 8 * (complex_vectors ? 2 : 1), cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
  });
}

int qmbed_gpu_operator_export_csr(qmbed_operator op, uint64_t* nnz_total, uint64_t* row_ptr, uint32_t* cols,
                                  double* values) {
  return guarded([&] {
    std::vector<uint64_t> rp;
    std::vector<uint32_t> c;
    std::vector<C64> v;
    op->op->export_csr(rp, c, v);
    if (nnz_total) *nnz_total = c.size();
    if (row_ptr) std::memcpy(row_ptr, rp.data(), rp.size() * sizeof(uint64_t));
    if (cols) std::memcpy(cols, c.data(), c.size() * sizeof(uint32_t));
    if (values)
      for (size_t i = 0; i < v.size(); ++i) {
        values[2 * i] = v[i].real();
        values[2 * i + 1] = v[i].imag();
      }
  });
}

int qmbed_gpu_operator_operand_bytes(qmbed_operator op, int precision, int complex_vectors, double* bytes) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(op->mu);
    *bytes = op->op->operand_bytes(precision, complex_vectors != 0);
  });
}

int qmbed_gpu_operator_set_lookup(qmbed_operator op, int mode) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(op->mu);
    op->op->set_lookup(mode);
  });
}

int qmbed_gpu_operator_lookup_info(qmbed_operator op, int* in_use, int* chain_form, uint64_t* table_bytes,
                                   double* table_seconds) {
  return guarded([&] {
    const ImageTable* t = op->op->basis().image_table();
    if (in_use) *in_use = op->op->lookup_in_use();
    if (chain_form) *chain_form = op->op->chain_form() && op->op->lookup_in_use() != 3 ? 1 : 0;
    if (table_bytes) *table_bytes = t ? t->bytes : 0;
    if (table_seconds) *table_seconds = t ? t->build_seconds : 0.0;
  });
}

namespace {

int run_eigsh(qmbed_operator op, const qmbed_eigsh_options* options, qmbed_eigsh_hint* hint, const double* initial,
              int n_initial, double* eigenvalues, double* residuals, double* eigenvectors, qmbed_eigsh_info* info) {
  return guarded([&] {
    if (!op || !options) raise(QMBED_INVALID_OPTIONS, "null operator or options");
    if (!eigenvalues || !residuals) raise(QMBED_INVALID_OPTIONS, "null eigenvalue or residual buffer");
    std::lock_guard<std::mutex> lock(op->mu);
    EigshOptions o;
    if (hint) {
      if (!std::isfinite(hint->lower) || !std::isfinite(hint->upper) || !std::isfinite(hint->gap))
        raise(QMBED_INVALID_OPTIONS, "eigsh hint must be finite");
      o.hint = true;
      o.hint_lower = hint->lower;
      o.hint_upper = hint->upper;
      o.hint_gap = hint->gap;
      o.hint_check_steps = hint->check_steps > 0 ? hint->check_steps : 8;
      o.restart_keep = hint->restart_keep;
    }
    o.eigenpairs = options->eigenpairs;
    o.target = options->target;
    o.shift = options->shift;
    o.krylov_dimension = options->krylov_dimension;
    o.tolerance = options->tolerance;
    o.max_iterations = options->max_iterations;
    o.seed = options->seed;
    o.want_vectors = eigenvectors != nullptr;
    const uint64_t n = op->op->dim();
    if (n_initial < 0 || (n_initial > 0 && !initial)) raise(QMBED_INVALID_OPTIONS, "invalid initial vectors");
    LinearOperatorView view = op->view();
    EigshResult r = eigsh(view, o, initial, n_initial, options->mode, op->block_ops());
    for (size_t i = 0; i < r.eigenvalues.size(); ++i) {
      eigenvalues[i] = r.eigenvalues[i];
      residuals[i] = r.residuals[i];
    }
    if (eigenvectors) {
      const size_t k = r.eigenvalues.size();
      BlockOps& ops = op->block_ops();
      if (r.complex_vectors) {
        QMBED_CUDA(cudaMemcpyAsync(eigenvectors, r.vectors.get(), k * n * 16, cudaMemcpyDeviceToHost, ops.stream()));
      } else {
        // widen to interleaved complex on the device, then one copy into the caller's buffer
        DeviceBuffer wide(std::max<size_t>(k * n, 1) * 16);
        ops.widen_real(r.vectors.as<double>(), wide.as<double>(), k * n);
        QMBED_CUDA(cudaMemcpyAsync(eigenvectors, wide.get(), k * n * 16, cudaMemcpyDeviceToHost, ops.stream()));
        ops.sync();
      }
      ops.sync();
    }
    if (info) {
      info->iterations = r.iterations;
      info->reorthogonalization_passes = r.reorthogonalization_passes;
      info->conditional_second_passes = r.conditional_second_passes;
      info->fp32_iterations = r.fp32_iterations;
      info->fp64_iterations = r.fp64_iterations;
      info->operator_applications = r.operator_applications;
      info->converged = r.converged ? 1 : 0;
      info->complex_vectors = r.complex_vectors ? 1 : 0;
    }
    if (hint) {
      hint->used = r.hint_used;
      hint->bound_applications = r.bound_applications;
    }
  });
}

}  // namespace

int qmbed_gpu_eigsh(qmbed_operator op, const qmbed_eigsh_options* options, const double* initial, int n_initial,
                    double* eigenvalues, double* residuals, double* eigenvectors, qmbed_eigsh_info* info) {
  return run_eigsh(op, options, nullptr, initial, n_initial, eigenvalues, residuals, eigenvectors, info);
}

int qmbed_gpu_eigsh_hinted(qmbed_operator op, const qmbed_eigsh_options* options, qmbed_eigsh_hint* hint,
                           const double* initial, int n_initial, double* eigenvalues, double* residuals,
                           double* eigenvectors, qmbed_eigsh_info* info) {
  return run_eigsh(op, options, hint, initial, n_initial, eigenvalues, residuals, eigenvectors, info);
}

int qmbed_gpu_expm_plan(qmbed_operator op, double coef_re, double coef_im, uint64_t max_degree, double tolerance,
                        uint64_t max_substeps, uint64_t* degree, uint64_t* scaling, double* shift, double* one_norm) {
  return guarded([&] {
    ExpmPlan plan = make_expm_plan(*op->op, C64(coef_re, coef_im), max_degree, tolerance, max_substeps);
    if (degree) *degree = plan.degree;
    if (scaling) *scaling = plan.scaling;
    if (shift) {
      shift[0] = plan.shift.real();
      shift[1] = plan.shift.imag();
    }
    if (one_norm) *one_norm = plan.one_norm;
  });
}

int qmbed_gpu_expm_apply_host(qmbed_operator op, double coef_re, double coef_im, uint64_t max_degree,
                              double tolerance, uint64_t max_substeps, int precision, const double* input,
                              double* output, uint64_t n_vectors) {
  return guarded([&] {
    if (precision != 64 && precision != 32) raise(QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
    std::lock_guard<std::mutex> lock(op->mu);
    ExpmPlan plan = make_expm_plan(*op->op, C64(coef_re, coef_im), max_degree, tolerance, max_substeps);
    const uint64_t n = op->op->dim();
    BlockOps& ops = op->block_ops();
    LinearOperatorView view = op->view();
    DeviceBuffer state64(std::max<uint64_t>(n, 1) * 16), state(std::max<uint64_t>(n, 1) * (precision == 64 ? 16 : 8));
    for (uint64_t k = 0; k < n_vectors; ++k) {
      QMBED_CUDA(cudaMemcpyAsync(state64.get(), input + 2 * k * n, n * 16, cudaMemcpyHostToDevice, ops.stream()));
      ops.convert(state64.get(), 64, state.get(), precision, 2 * n);
      expm_apply(plan, view, state.get(), precision, ops);
      ops.convert(state.get(), precision, state64.get(), 64, 2 * n);
      QMBED_CUDA(cudaMemcpyAsync(output + 2 * k * n, state64.get(), n * 16, cudaMemcpyDeviceToHost, ops.stream()));
      ops.sync();
    }
  });
}

int qmbed_gpu_evolve(qmbed_operator op, const double* initial, int n_times, const double* times,
                     uint64_t krylov_dimension, double tolerance, uint64_t max_substeps, double* states,
                     double* diagnostics) {
  return guarded([&] {
    if (!initial || !states || n_times < 0 || (n_times > 0 && !times))
      raise(QMBED_INVALID_OPTIONS, "evolution needs an initial state, a time grid and an output array");
    std::lock_guard<std::mutex> lock(op->mu);
    EvolutionOptions o;
    o.times.assign(times, times + n_times);
    o.krylov_dimension = krylov_dimension;
    o.tolerance = tolerance;
    o.max_substeps = max_substeps;
    EvolutionDiagnostics d;
    evolve(op->view(), initial, o, states, d, op->block_ops());
    if (diagnostics) {
      const double fields[7] = {static_cast<double>(d.lanczos_projections), static_cast<double>(d.matrix_vector_products),
                                static_cast<double>(d.real_lanczos_projections),
                                static_cast<double>(d.real_matrix_vector_products),
                                static_cast<double>(d.accepted_substeps), static_cast<double>(d.rejected_trial_intervals),
                                d.maximum_estimated_error};
      for (int i = 0; i < 7; ++i) diagnostics[i] = fields[i];
    }
  });
}

int qmbed_gpu_expm_lanczos(qmbed_operator op, const double* initial, double time, uint64_t krylov_dimension,
                           double* out) {
  return guarded([&] {
    if (!initial || !out) raise(QMBED_INVALID_OPTIONS, "expm_lanczos needs input and output vectors");
    std::lock_guard<std::mutex> lock(op->mu);
    expm_lanczos(op->view(), initial, time, krylov_dimension, out, op->block_ops());
  });
}

int qmbed_gpu_chebyshev_evolve_device(qmbed_operator op, double* state, int n_times, const double* times,
                                      double e_min, double e_max, double tolerance, int precision, double* info) {
  return guarded([&] {
    if (!state || n_times <= 0 || !times)
      raise(QMBED_INVALID_OPTIONS, "evolution needs a device state and a time grid");
    std::lock_guard<std::mutex> lock(op->mu);
    if (std::isnan(e_min) && std::isnan(e_max)) flip_chain_norm_bounds(*op->op, &e_min, &e_max);
    ChebyshevInfo ci;
    chebyshev_evolve_device(*op->op, state, std::vector<double>(times, times + n_times), e_min, e_max, tolerance,
                            precision, ci, op->block_ops());
    if (info) {
      info[0] = static_cast<double>(ci.applications);
      info[1] = static_cast<double>(ci.intervals);
      info[2] = ci.e_min;
      info[3] = ci.e_max;
      info[4] = ci.max_norm_drift;
    }
  });
}

int qmbed_gpu_chebyshev_evolve(qmbed_operator op, const double* initial, int n_times, const double* times,
                               double e_min, double e_max, double tolerance, int precision, int final_only,
                               double* states, double* info) {
  return guarded([&] {
    if (!initial || !states || n_times < 0 || (n_times > 0 && !times))
      raise(QMBED_INVALID_OPTIONS, "evolution needs an initial state, a time grid and an output array");
    std::lock_guard<std::mutex> lock(op->mu);
    if (std::isnan(e_min) && std::isnan(e_max)) flip_chain_norm_bounds(*op->op, &e_min, &e_max);
    ChebyshevInfo ci;
    chebyshev_evolve(*op->op, initial, std::vector<double>(times, times + n_times), e_min, e_max, tolerance, precision,
                     final_only != 0, states, ci, op->block_ops());
    if (info) {
      info[0] = static_cast<double>(ci.applications);
      info[1] = static_cast<double>(ci.intervals);
      info[2] = ci.e_min;
      info[3] = ci.e_max;
      info[4] = ci.max_norm_drift;
    }
  });
}

int qmbed_gpu_scan_solve(int n_sectors, int n_components, const qmbed_operator* components, int n_points,
                         const double* coefficients, int eigenpairs, double tolerance, int max_steps, uint64_t seed,
                         double* eigenvalues, double* residuals, double* e_max, int* steps, double* info) {
  return guarded([&] {
    if (n_sectors < 1 || n_components < 1 || !components || !coefficients || !eigenvalues || !steps)
      raise(QMBED_INVALID_OPTIONS, "a scan needs sectors, components, coefficients and outputs");
    std::vector<std::vector<const SpinOperator*>> comps(static_cast<size_t>(n_sectors));
    for (int s = 0; s < n_sectors; ++s)
      for (int k = 0; k < n_components; ++k) {
        const qmbed_operator c = components[s * n_components + k];
        if (!c) raise(QMBED_INVALID_OPTIONS, "null scan component");
        comps[s].push_back(c->op.get());
      }
    qmbed_operator_s& first = *components[0];
    std::lock_guard<std::mutex> lock(first.mu);
    QMBED_CUDA(cudaSetDevice(first.op->basis().device()));
    const ScanResult r = scan_lowest(comps, std::vector<double>(coefficients, coefficients + n_points * n_components),
                                     n_points, eigenpairs, tolerance, max_steps, seed, first.block_ops());
    std::copy(r.eigenvalues.begin(), r.eigenvalues.end(), eigenvalues);
    std::copy(r.steps.begin(), r.steps.end(), steps);
    if (residuals) std::copy(r.residuals.begin(), r.residuals.end(), residuals);
    if (e_max) std::copy(r.e_max.begin(), r.e_max.end(), e_max);
    if (info) {
      info[0] = static_cast<double>(r.total_steps);
      info[1] = static_cast<double>(r.applications);
      info[2] = static_cast<double>(r.applications_verification);
      info[3] = r.graph ? 1.0 : 0.0;
      info[4] = r.pass1_seconds;
      info[5] = r.seconds;
      info[6] = r.max_relative_residual;
      info[7] = static_cast<double>(r.merged_copies);
      info[8] = static_cast<double>(r.tuned_blocks_per_sm);
      info[9] = r.tuning_ms.empty() ? 0.0 : *std::min_element(r.tuning_ms.begin(), r.tuning_ms.end());
      info[10] = static_cast<double>(r.tuned_rows_per_warp);
    }
  });
}

int qmbed_gpu_scan_lowest(int n_sectors, int n_components, const qmbed_operator* components, int n_points,
                          const double* coefficients, int eigenpairs, double tolerance, int max_steps, uint64_t seed,
                          double* eigenvalues, int* steps, double* info) {
  double full[11] = {0};
  const int rc = qmbed_gpu_scan_solve(n_sectors, n_components, components, n_points, coefficients, eigenpairs,
                                      tolerance, max_steps, seed, eigenvalues, nullptr, nullptr, steps, full);
  if (rc == QMBED_STATUS_OK && info) {
    info[0] = full[0];
    info[1] = full[1];
  }
  return rc;
}

int qmbed_gpu_flip_wait_selftest(int device, int* status) {
  return guarded([&] {
    if (!status) raise(QMBED_INVALID_OPTIONS, "null status");
    *status = flip_stage_wait_selftest(device);
  });
}

int qmbed_gpu_scan_barrier_selftest(int device, int* status) {
  return guarded([&] {
    if (!status) raise(QMBED_INVALID_OPTIONS, "null status");
    *status = scan_barrier_selftest(device);
  });
}

int qmbed_gpu_lanczos_extremes(qmbed_operator op, int steps, uint64_t seed, double* out) {
  return guarded([&] {
    if (!op || !out) raise(QMBED_INVALID_OPTIONS, "null operator or output");
    std::lock_guard<std::mutex> lock(op->mu);
    const RitzExtremes r = lanczos_extremes(op->view(), steps, seed, op->block_ops());
    out[0] = r.min;
    out[1] = r.max;
    out[2] = r.min_residual;
    out[3] = r.max_residual;
  });
}

struct qmbed_mlp_s {
  std::unique_ptr<Mlp> net;
  std::mutex mu;
};

int qmbed_gpu_mlp_create(int device, int inputs, int outputs, int width, int hidden_layers, uint64_t seed,
                         qmbed_mlp* out) {
  return guarded([&] {
    auto h = std::make_unique<qmbed_mlp_s>();
    h->net = std::make_unique<Mlp>(device, inputs, outputs, width, hidden_layers, seed);
    *out = h.release();
  });
}

int qmbed_gpu_mlp_destroy(qmbed_mlp mlp) {
  return guarded([&] { delete mlp; });
}

int qmbed_gpu_mlp_parameter_count(qmbed_mlp mlp, uint64_t* count) {
  return guarded([&] { *count = mlp->net->parameter_count(); });
}

int qmbed_gpu_mlp_get_parameters(qmbed_mlp mlp, float* out) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    mlp->net->get_parameters(out);
  });
}

int qmbed_gpu_mlp_set_parameters(qmbed_mlp mlp, const float* in) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    mlp->net->set_parameters(in);
  });
}

int qmbed_gpu_mlp_set_scaling(qmbed_mlp mlp, const float* in_mean, const float* in_std, const float* out_mean,
                              const float* out_std) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    const int ni = mlp->net->inputs(), no = mlp->net->outputs();
    mlp->net->set_scaling(std::vector<float>(in_mean, in_mean + ni), std::vector<float>(in_std, in_std + ni),
                          std::vector<float>(out_mean, out_mean + no), std::vector<float>(out_std, out_std + no));
  });
}

int qmbed_gpu_mlp_get_scaling(qmbed_mlp mlp, float* in_mean, float* in_std, float* out_mean, float* out_std) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    mlp->net->get_scaling(in_mean, in_std, out_mean, out_std);
  });
}

int qmbed_gpu_mlp_gradients(qmbed_mlp mlp, const float* X, const float* Y, int n, float* grads, float* loss) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    const float l = mlp->net->gradients(X, Y, n, grads);
    if (loss) *loss = l;
  });
}

int qmbed_gpu_mlp_train(qmbed_mlp mlp, const float* X, const float* Y, int n, int epochs, int batch,
                        float learning_rate, uint64_t seed, float* loss) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    const float l = mlp->net->train(X, Y, n, epochs, batch, learning_rate, seed);
    if (loss) *loss = l;
  });
}

int qmbed_gpu_mlp_predict(qmbed_mlp mlp, const float* X, int n, float* Y) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(mlp->mu);
    mlp->net->predict(X, n, Y);
  });
}



int qmbed_gpu_lanczos_create(qmbed_operator op, const double* initial, uint64_t krylov_dimension, double tolerance,
                             qmbed_lanczos* out) {
  return guarded([&] {
    if (!out) raise(QMBED_INVALID_OPTIONS, "lanczos_create needs an output handle");
    auto h = std::make_unique<qmbed_lanczos_s>();
    {
      std::lock_guard<std::mutex> lock(op->mu);
      lanczos_ritz(op->view(), initial, krylov_dimension, tolerance, h->d, op->block_ops());
    }
    *out = h.release();
  });
}

int qmbed_gpu_lanczos_destroy(qmbed_lanczos lanczos) {
  return guarded([&] { delete lanczos; });
}

int qmbed_gpu_lanczos_info(qmbed_lanczos l, uint64_t* dimension, uint64_t* krylov_dimension, double* initial_norm,
                           int* is_real, uint64_t* second_passes) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    if (dimension) *dimension = l->d.n;
    if (krylov_dimension) *krylov_dimension = static_cast<uint64_t>(l->d.size);
    if (initial_norm) *initial_norm = l->d.initial_norm;
    if (is_real) *is_real = l->d.real ? 1 : 0;
    if (second_passes) *second_passes = static_cast<uint64_t>(l->d.second_passes);
  });
}

int qmbed_gpu_lanczos_ritz(qmbed_lanczos l, double* values, double* vectors, double* diagonal, double* off_diagonal) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    const int m = l->d.size;
    for (int c = 0; c < m; ++c) {
      if (values) values[c] = l->d.eigenvalues[c];
      if (vectors)
        for (int r = 0; r < m; ++r) vectors[static_cast<size_t>(c) * m + r] = l->d.vec(r, c);
      if (diagonal) diagonal[c] = l->d.diagonal[c];
      if (off_diagonal && c + 1 < m) off_diagonal[c] = l->d.off_diagonal[c];
    }
  });
}

int qmbed_gpu_lanczos_basis(qmbed_lanczos l, double* basis) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    QMBED_CUDA(cudaSetDevice(l->d.device));
    for (int j = 0; j < l->d.size; ++j) {
      const std::vector<double> col = lanczos_column_host(l->d, j);
      std::memcpy(basis + 2 * static_cast<size_t>(j) * l->d.n, col.data(), col.size() * sizeof(double));
    }
  });
}

int qmbed_gpu_lanczos_combine(qmbed_lanczos l, const double* coefficients, double* out) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    if (!coefficients || !out) raise(QMBED_INVALID_OPTIONS, "linear combination needs coefficients and an output");
    std::vector<C64> c(static_cast<size_t>(l->d.size));
    for (int b = 0; b < l->d.size; ++b) c[b] = C64(coefficients[2 * b], coefficients[2 * b + 1]);
    lanczos_vector_out(*l, c, out);
  });
}

int qmbed_gpu_lanczos_exponential(qmbed_lanczos l, double coefficient_re, double coefficient_im, double* out) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    if (!out) raise(QMBED_INVALID_OPTIONS, "exponential action needs an output vector");
    lanczos_vector_out(*l, exponential_coefficients(l->d, C64(coefficient_re, coefficient_im)), out);
  });
}

int qmbed_gpu_lanczos_thermal(qmbed_lanczos l, int method, int n_betas, const double* betas, int n_observables,
                              const qmbed_operator* observables, double* values, double* identity) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    if (method != 0 && method != 1) raise(QMBED_INVALID_OPTIONS, "thermal method must be FTLM (0) or LTLM (1)");
    if (n_observables <= 0 || !observables) raise(QMBED_INVALID_OPTIONS, "thermal observables must be nonempty");
    const std::vector<double> grid = beta_grid(n_betas, betas);
    std::vector<std::vector<C64>> projected;
    for (int o = 0; o < n_observables; ++o) {
      qmbed_operator_s& a = *observables[o];
      std::lock_guard<std::mutex> alock(a.mu);
      projected.push_back(project_observable(l->d, a.view(), method == 1, a.block_ops()));
    }
    std::vector<std::vector<C64>> out;
    std::vector<double> id;
    thermal_contraction(method == 1, l->d.eigenvalues, ritz_columns(l->d), projected, grid, out, id);
    for (size_t o = 0; o < out.size(); ++o)
      for (size_t b = 0; b < grid.size(); ++b) {
        values[2 * (o * grid.size() + b)] = out[o][b].real();
        values[2 * (o * grid.size() + b) + 1] = out[o][b].imag();
      }
    for (size_t b = 0; b < grid.size(); ++b) identity[b] = id[b];
  });
}

int qmbed_gpu_lanczos_project(qmbed_lanczos l, int method, qmbed_operator observable, double* matrix_elements) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(l->mu);
    if (method != 0 && method != 1) raise(QMBED_INVALID_OPTIONS, "thermal method must be FTLM (0) or LTLM (1)");
    if (!observable || !matrix_elements) raise(QMBED_INVALID_OPTIONS, "projection needs an observable and an output");
    std::lock_guard<std::mutex> alock(observable->mu);
    const std::vector<C64> p = project_observable(l->d, observable->view(), method == 1, observable->block_ops());
    for (size_t i = 0; i < p.size(); ++i) {
      matrix_elements[2 * i] = p[i].real();
      matrix_elements[2 * i + 1] = p[i].imag();
    }
  });
}

int qmbed_gpu_thermal_contraction(int method, int m, const double* eigenvalues, const double* eigenvectors,
                                  int n_observables, const double* matrix_elements, int n_betas, const double* betas,
                                  double* values, double* identity) {
  return guarded([&] {
    if (method != 0 && method != 1) raise(QMBED_INVALID_OPTIONS, "thermal method must be FTLM (0) or LTLM (1)");
    if (m < 0 || n_observables < 0 || (m > 0 && (!eigenvalues || !eigenvectors)))
      raise(QMBED_DIMENSION_MISMATCH, "thermal Lanczos contraction requires a finite square Ritz eigensystem");
    const std::vector<double> grid = beta_grid(n_betas, betas);
    std::vector<double> e(eigenvalues, eigenvalues + m);
    std::vector<std::vector<double>> columns(static_cast<size_t>(m), std::vector<double>(static_cast<size_t>(m)));
    for (int c = 0; c < m; ++c)
      for (int r = 0; r < m; ++r) columns[c][r] = eigenvectors[static_cast<size_t>(r) * m + c];
    const size_t per = method == 1 ? static_cast<size_t>(m) * m : static_cast<size_t>(m);
    std::vector<std::vector<C64>> projected(static_cast<size_t>(n_observables), std::vector<C64>(per));
    for (int o = 0; o < n_observables; ++o)
      for (size_t i = 0; i < per; ++i)
        projected[o][i] = C64(matrix_elements[2 * (o * per + i)], matrix_elements[2 * (o * per + i) + 1]);
    std::vector<std::vector<C64>> out;
    std::vector<double> id;
    thermal_contraction(method == 1, e, columns, projected, grid, out, id);
    for (size_t o = 0; o < out.size(); ++o)
      for (size_t b = 0; b < grid.size(); ++b) {
        values[2 * (o * grid.size() + b)] = out[o][b].real();
        values[2 * (o * grid.size() + b) + 1] = out[o][b].imag();
      }
    for (size_t b = 0; b < grid.size(); ++b) identity[b] = id[b];
  });
}

int qmbed_gpu_thermal_iteration(qmbed_operator op, const double* initial, int n_betas, const double* betas,
                                uint64_t krylov_dimension, double tolerance, double* log_partition,
                                double* mean_energy, uint64_t* krylov_out) {
  return guarded([&] {
    validate_lanczos(krylov_dimension, tolerance);
    const std::vector<double> grid = beta_grid(n_betas, betas);
    std::lock_guard<std::mutex> lock(op->mu);
    // validate the temperatures before the recurrence runs (src/solve/mod.rs:3473-3482)
    bool ok = !grid.empty();
    for (double b : grid) ok = ok && std::isfinite(b) && b >= 0.0;
    if (!ok) raise(QMBED_INVALID_OPTIONS, "inverse temperatures must be nonempty, finite, and nonnegative");
    LanczosDecomposition d;
    lanczos_ritz(op->view(), initial, krylov_dimension, tolerance, d, op->block_ops());
    const ThermalEstimate t = thermal_estimate(d, op->op->dim(), grid);
    for (size_t b = 0; b < grid.size(); ++b) {
      log_partition[b] = t.log_partition[b];
      mean_energy[b] = t.mean_energy[b];
    }
    if (krylov_out) *krylov_out = static_cast<uint64_t>(t.krylov_dimension);
  });
}

int qmbed_gpu_ftlm_sample(qmbed_operator op, int n_vectors, uint64_t seed, int n_betas, const double* betas,
                          uint64_t krylov_dimension, double tolerance, double* log_partition, double* mean_energy,
                          int* lengths) {
  return guarded([&] {
    const std::vector<double> grid = beta_grid(n_betas, betas);
    std::lock_guard<std::mutex> lock(op->mu);
    std::vector<double> lz, e;
    std::vector<int> len;
    ftlm_sample(op->view(), n_vectors, seed, krylov_dimension, tolerance, grid, lz, e, len, op->block_ops());
    std::copy(lz.begin(), lz.end(), log_partition);
    std::copy(e.begin(), e.end(), mean_energy);
    if (lengths) std::copy(len.begin(), len.end(), lengths);
  });
}

int qmbed_gpu_ftlm_start(qmbed_operator op, uint64_t seed, int index, double* out) {
  return guarded([&] {
    if (!out || index < 0) raise(QMBED_INVALID_OPTIONS, "start vector needs a nonnegative index and an output");
    std::lock_guard<std::mutex> lock(op->mu);
    const LinearOperatorView view = op->view();
    BlockOps& ops = op->block_ops();
    const uint64_t n = view.dim;
    DeviceBuffer v(std::max<uint64_t>(n, 1) * 16), wide(std::max<uint64_t>(n, 1) * 16);
    ftlm_start_vector(view, seed, index, v.as<double>(), ops);
    if (view.real) ops.widen_real(v.as<double>(), wide.as<double>(), n);
    QMBED_CUDA(cudaMemcpyAsync(out, view.real ? wide.get() : v.get(), n * 16, cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
  });
}

struct qmbed_shift_s {
  std::shared_ptr<SpinBasis> target;
  std::shared_ptr<SpinOperator> terms;  // on the source basis
  cudaStream_t stream = nullptr;
  std::unique_ptr<BlockOps> ops;
  std::mutex mu;
  ~qmbed_shift_s() {
    ops.reset();
    if (stream) cudaStreamDestroy(stream);
  }
  BlockOps& block_ops() {
    if (!ops) {
      QMBED_CUDA(cudaSetDevice(target->device()));
      QMBED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      ops = std::make_unique<BlockOps>(target->device(), stream);
    }
    return *ops;
  }
};

int qmbed_gpu_shift_create(qmbed_basis source, qmbed_basis target, int n_terms, const int* arity, const char* symbols,
                           const int* n_couplings, const double* coefficients, const int* sites, qmbed_shift* out) {
  return guarded([&] {
    if (!source || !target || !out) raise(QMBED_INVALID_OPTIONS, "a sector shift needs two bases and an output");
    auto terms = decode_terms(n_terms, arity, symbols, n_couplings, coefficients, sites);
    OperatorChecks checks;
    checks.hermiticity = false;
    checks.particle_conservation = false;
    auto h = std::make_unique<qmbed_shift_s>();
    h->target = target->basis;
    h->terms = std::make_shared<SpinOperator>(source->basis, terms, checks, kStorageMatrixFree);
    if (h->target->sites() != source->basis->sites() || h->target->device() != source->basis->device())
      raise(QMBED_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
    *out = h.release();
  });
}

int qmbed_gpu_shift_destroy(qmbed_shift shift) {
  return guarded([&] { delete shift; });
}

int qmbed_gpu_shift_apply_device(qmbed_shift shift, const double* x, double* y, void* stream) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(shift->mu);
    shift->terms->apply_shift(*shift->target, x, y, static_cast<cudaStream_t>(stream));
  });
}

int qmbed_gpu_shift_apply_host(qmbed_shift shift, uint64_t n_input, const double* x, uint64_t n_output, double* y) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(shift->mu);
    const uint64_t ns = shift->terms->dim(), nt = shift->target->dim();
    if (n_input != ns || n_output != nt)
      raise(QMBED_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
    BlockOps& ops = shift->block_ops();
    DeviceBuffer dx(std::max<uint64_t>(ns, 1) * 16), dy(std::max<uint64_t>(nt, 1) * 16);
    QMBED_CUDA(cudaMemcpyAsync(dx.get(), x, ns * 16, cudaMemcpyHostToDevice, ops.stream()));
    shift->terms->apply_shift(*shift->target, dx.as<double>(), dy.as<double>(), ops.stream());
    QMBED_CUDA(cudaMemcpyAsync(y, dy.get(), nt * 16, cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
  });
}

int qmbed_gpu_spectral_function(qmbed_operator target, qmbed_shift probe, uint64_t n_source, const double* source,
                                int n_frequencies, const double* frequencies, double reference_energy,
                                double broadening, uint64_t krylov_dimension, double tolerance, double* out) {
  return guarded([&] {
    if (!target || !probe || !source || !out || n_frequencies < 0 || (n_frequencies > 0 && !frequencies))
      raise(QMBED_INVALID_OPTIONS, "a spectrum needs a target Hamiltonian, a probe, a source and a frequency grid");
    SpectrumOptions o;
    o.frequencies.assign(frequencies, frequencies + n_frequencies);
    o.reference_energy = reference_energy;
    o.broadening = broadening;
    o.krylov_dimension = krylov_dimension;
    o.tolerance = tolerance;
    validate_spectrum(o);
    std::lock_guard<std::mutex> lock(target->mu);
    std::lock_guard<std::mutex> plock(probe->mu);
    const uint64_t nt = target->op->dim(), ns = probe->terms->dim();
    // the probe must land in the target Hamiltonian's sector
    const SectorParams& a = probe->target->params();
    const SectorParams& b = target->op->basis().params();
    const bool same = a.sites == b.sites && a.up == b.up && a.has_momentum == b.has_momentum &&
                      a.momentum == b.momentum && a.parity == b.parity && a.inversion == b.inversion &&
                      probe->target->normalization() == target->op->basis().normalization();
    if (!same || probe->target->dim() != nt || n_source != ns)
      raise(QMBED_DIMENSION_MISMATCH, "target Hamiltonian, source, and probe shapes are incompatible");
    BlockOps& ops = target->block_ops();
    DeviceBuffer dx(std::max<uint64_t>(ns, 1) * 16), created(std::max<uint64_t>(nt, 1) * 16);
    QMBED_CUDA(cudaMemcpyAsync(dx.get(), source, ns * 16, cudaMemcpyHostToDevice, ops.stream()));
    probe->terms->apply_shift(*probe->target, dx.as<double>(), created.as<double>(), ops.stream());
    const std::vector<double> r = spectral_function(target->view(), created.as<double>(), o, ops);
    std::copy(r.begin(), r.end(), out);
  });
}

int qmbed_gpu_deterministic_start(int device, uint64_t n, uint64_t seed, double* out) {
  return guarded([&] {
    QMBED_CUDA(cudaSetDevice(device));
    cudaStream_t stream;
    QMBED_CUDA(cudaStreamCreate(&stream));
    {
      BlockOps ops(device, stream);
      DeviceBuffer v(std::max<uint64_t>(n, 1) * 8);
      ops.lcg_start(v.get(), n, seed, 64, false);
      const double norm = ops.norm(v.get(), n, 64, false);
      if (!std::isfinite(norm) || norm <= 2.220446049250313e-16) raise_nonconvergence(0, norm);
      ops.scale(v.get(), n, norm, 64, false);
      QMBED_CUDA(cudaMemcpyAsync(out, v.get(), n * 8, cudaMemcpyDeviceToHost, stream));
      ops.sync();
    }
    cudaStreamDestroy(stream);
  });
}

char* qmbed_run_json(const char* request) { return to_c_string(respond(request, false)); }

char* qmbed_command_json(const char* request) { return to_c_string(respond(request, true)); }

void qmbed_string_free(char* response) { std::free(response); }

// run_drive_evolution_json / execute_drive_evolution (bindings/capi/src/lib.rs:2206-2225, 4695-4746):
// the model's static part and components, coefficients from the caller's
// callback at every internal time, the adaptive RK4 of evolve_time_dependent.
char* qmbed_evolve_model_with_drive_json(const char* request, void* callback, void* context) {
  if (!request) return to_c_string(R"({"status":"error","error":"request pointer is null"})");
  if (!callback) return to_c_string(R"({"status":"error","error":"drive callback is null"})");
  return json_call(request, [callback, context](const Value& r) { return drive_evolution(r, callback, context); });
}

char* qmbed_register_user_basis_32_json(const char* request, void* op, void* next_state, void* pre_check, void* maps,
                                        size_t n_maps) {
  (void)request, (void)op, (void)next_state, (void)pre_check, (void)maps, (void)n_maps;
  return to_c_string(R"({"status":"error","error":"unsupported backend: user bases are outside the GPU engine"})");
}

char* qmbed_register_user_basis_64_json(const char* request, void* op, void* next_state, void* pre_check, void* maps,
                                        size_t n_maps) {
  (void)request, (void)op, (void)next_state, (void)pre_check, (void)maps, (void)n_maps;
  return to_c_string(R"({"status":"error","error":"unsupported backend: user bases are outside the GPU engine"})");
}

}  // extern "C"
