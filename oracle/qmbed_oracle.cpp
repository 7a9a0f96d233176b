// QMBED spin-chain hot path: CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This file restates, in plain C++17, the algorithms
// of the Rust reference (matrixlab-research/QMBED) for the symmetry-reduced
// spin-1/2 chain Hamiltonian and the solvers on it. Only the test suite, the
// smoke check and the CPU-baseline leg of the benchmark load it; the product
// library under qmbed_b200/ never links, calls or falls back to it.
//
// Every function names the reference file:line it follows. The reference
// cannot be built here (no Rust toolchain), so parity of this oracle is pinned
// against the known answers held in the reference's own tests (see
// tests/golden/reference_anchors.json) and against independent dense
// numpy/scipy computations in tests/test_oracle_*.py.
//
// Third-party arithmetic: the reference diagonalises projected/tridiagonal
// matrices with nalgebra 0.33.3 `SymmetricEigen` and dense Hermitian matrices
// with faer 0.24.4. Neither crate is present. This oracle uses its own
// implicit-QL (tridiagonal) and cyclic Jacobi (dense Hermitian) solvers, which
// agree at eigenvalue level; eigenvector signs/phases are not bitwise equal.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

using u128 = unsigned __int128;
using C64 = std::complex<double>;
constexpr double EPS = std::numeric_limits<double>::epsilon();

// ----------------------------------------------------------------------------
// Errors: categories and Display texts of `QmbedError` (src/error.rs:4-35).
// ----------------------------------------------------------------------------
enum ErrorCode {
  ERR_OK = 0,
  ERR_INVALID_OPERATOR = 1,
  ERR_INVALID_COUPLING = 2,
  ERR_INVALID_SITE = 3,
  ERR_STATE_NOT_IN_BASIS = 4,
  ERR_INVALID_SECTOR = 5,
  ERR_INCOMPATIBLE_SYMMETRY = 6,
  ERR_NON_HERMITIAN = 7,
  ERR_INVALID_OPTIONS = 8,
  ERR_DIMENSION_MISMATCH = 9,
  ERR_RANK_DEFICIENT = 10,
  ERR_UNSUPPORTED_BACKEND = 11,
  ERR_INTERNAL_STATE = 13,
  ERR_NON_CONVERGENCE = 14,
};

struct QError : std::runtime_error {
  int code;
  double residual = 0.0;
  size_t iterations = 0;
  QError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& detail) {
  std::string text;
  switch (code) {
    case ERR_INVALID_OPERATOR: text = "invalid or unregistered operator: " + detail; break;
    case ERR_INVALID_COUPLING: text = "invalid coupling: " + detail; break;
    case ERR_INVALID_SITE: text = detail; break;
    case ERR_STATE_NOT_IN_BASIS: text = "state is not represented by this basis"; break;
    case ERR_INVALID_SECTOR: text = "invalid Hilbert-space sector: " + detail; break;
    case ERR_INCOMPATIBLE_SYMMETRY: text = "incompatible symmetry request: " + detail; break;
    case ERR_NON_HERMITIAN: text = "a Hermitian operator is required"; break;
    case ERR_INVALID_OPTIONS: text = "invalid options: " + detail; break;
    case ERR_DIMENSION_MISMATCH: text = "dimension mismatch: " + detail; break;
    case ERR_UNSUPPORTED_BACKEND: text = "unsupported backend: " + detail; break;
    case ERR_INTERNAL_STATE: text = "internal state error: " + detail; break;
    default: text = detail; break;
  }
  throw QError(code, text);
}

[[noreturn]] void fail_nonconvergence(size_t iterations, double residual) {
  char buffer[160];
  // Rust `{:e}` prints the shortest round-trip mantissa; %.17g is close enough
  // for a test oracle (the text is not compared byte for byte).
  std::snprintf(buffer, sizeof(buffer),
                "solver did not converge after %zu iterations; residual=%.6e", iterations,
                residual);
  QError error(ERR_NON_CONVERGENCE, buffer);
  error.iterations = iterations;
  error.residual = residual;
  throw error;
}

struct U128Hash {
  size_t operator()(u128 value) const noexcept {
    uint64_t lo = static_cast<uint64_t>(value);
    uint64_t hi = static_cast<uint64_t>(value >> 64);
    uint64_t x = lo ^ (hi * 0x9e3779b97f4a7c15ULL);
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return static_cast<size_t>(x);
  }
};

// binomial (src/basis/mod.rs:6217-6222)
size_t binomial(size_t n, size_t k) {
  size_t kk = std::min(k, n >= k ? n - k : 0);
  if (k > n) return 0;
  size_t value = 1;
  for (size_t index = 0; index < kk; ++index) value = value * (n - index) / (index + 1);
  return value;
}

// fixed_weight_states: Gosper's hack in colex order (src/basis/mod.rs:373-424)
std::vector<u128> fixed_weight_states(size_t sites, long particles) {
  if (sites > 128) fail(ERR_UNSUPPORTED_BACKEND, "the initial u128 state backend supports at most 128 orbitals");
  if (particles >= 0 && static_cast<size_t>(particles) > sites)
    fail(ERR_INVALID_SECTOR, "particle count exceeds site count");
  std::vector<u128> states;
  if (particles < 0) {
    if (sites >= 48) fail(ERR_UNSUPPORTED_BACKEND, "enumerating the unconstrained Hilbert space is infeasible");
    u128 limit = static_cast<u128>(1) << sites;
    states.reserve(static_cast<size_t>(limit));
    for (u128 s = 0; s < limit; ++s) states.push_back(s);
    return states;
  }
  if (particles == 0) return {0};
  if (static_cast<size_t>(particles) == sites) {
    u128 state = sites == 128 ? ~static_cast<u128>(0) : ((static_cast<u128>(1) << sites) - 1);
    return {state};
  }
  u128 state = (static_cast<u128>(1) << particles) - 1;
  bool has_limit = sites < 128;
  u128 limit = has_limit ? (static_cast<u128>(1) << sites) : 0;
  states.reserve(binomial(sites, static_cast<size_t>(particles)));
  for (;;) {
    states.push_back(state);
    u128 low_bit = state & (~state + 1);
    u128 ripple = state + low_bit;
    if (ripple < state) break;  // checked_add overflow
    u128 next = (((ripple ^ state) >> 2) / low_bit) | ripple;
    if (has_limit && next >= limit) break;
    state = next;
  }
  return states;
}

int popcount128(u128 v) {
  return __builtin_popcountll(static_cast<uint64_t>(v)) +
         __builtin_popcountll(static_cast<uint64_t>(v >> 64));
}
int ctz128(u128 v) {
  uint64_t lo = static_cast<uint64_t>(v);
  if (lo) return __builtin_ctzll(lo);
  return 64 + __builtin_ctzll(static_cast<uint64_t>(v >> 64));
}

// fixed_weight_state_index: colex rank (src/basis/mod.rs:640-659)
bool fixed_weight_state_index(u128 state, size_t sites, size_t particles, size_t* out) {
  if (particles > sites || static_cast<size_t>(popcount128(state)) != particles ||
      (sites < 128 && state >= (static_cast<u128>(1) << sites)))
    return false;
  size_t rank = 0, ordinal = 1;
  u128 remaining = state;
  while (remaining != 0) {
    size_t position = static_cast<size_t>(ctz128(remaining));
    if (position >= ordinal) rank += binomial(position, ordinal);
    ordinal += 1;
    remaining &= remaining - 1;
  }
  *out = rank;
  return true;
}

// rotate_lattice_state, base 2 (src/basis/mod.rs:661-686)
u128 rotate_lattice_state(u128 state, size_t shift, size_t sites) {
  if (sites == 0) return state;
  shift %= sites;
  if (shift == 0) return state;
  u128 mask = sites == 128 ? ~static_cast<u128>(0) : ((static_cast<u128>(1) << sites) - 1);
  return ((state << shift) & mask) | (state >> (sites - shift));
}

// reflect_lattice_state, base 2 (src/basis/mod.rs:688-698)
u128 reflect_lattice_state(u128 state, size_t sites) {
  u128 reflected = 0;
  for (size_t site = 0; site < sites; ++site) {
    u128 digit = (state >> site) & 1;
    reflected += digit << (sites - site - 1);
  }
  return reflected;
}

struct SymmetryImage {
  u128 representative;
  C64 phase;
  size_t orbit_size;
};

// ----------------------------------------------------------------------------
// Spin-1/2 chain basis (SpinBasis1D, src/basis/mod.rs:1018-1035, 1312-1412)
// ----------------------------------------------------------------------------
struct SpinBasis {
  size_t sites = 0;
  long up = -1;  // -1: no fixed weight
  bool has_momentum = false;
  size_t momentum = 0;  // canonical k in [0, L)
  int parity = 0;       // 0: none, else +-1
  int normalization = 0;  // 0 angular momentum, 1 Pauli, 2 Pauli-Cartesian
  double z_factors[2];
  double raise_factors[2];
  double lower_factors[2];
  std::vector<u128> states;
  std::vector<size_t> orbit_lengths;
  std::unordered_map<u128, SymmetryImage, U128Hash> lookup;

  bool symmetric() const { return has_momentum || parity != 0; }
  size_t len() const { return states.size(); }

  // SpinBasis1D::index (src/basis/mod.rs:1429-1442); state_index 623-627;
  // direct_state_index 629-636.
  bool index(u128 state, size_t* out) const {
    if (!symmetric()) {
      if (up >= 0) return fixed_weight_state_index(state, sites, static_cast<size_t>(up), out);
      if (state >= static_cast<u128>(states.size())) return false;
      *out = static_cast<size_t>(state);
      return true;
    }
    auto it = std::lower_bound(states.begin(), states.end(), state);
    if (it == states.end() || *it != state) return false;
    *out = static_cast<size_t>(it - states.begin());
    return true;
  }

  // transition_orbit_size (src/basis/mod.rs:1529-1534)
  size_t transition_orbit_size(u128 state) const {
    if (!symmetric()) return 1;
    size_t index_value;
    if (!index(state, &index_value)) fail(ERR_STATE_NOT_IN_BASIS, "");
    return orbit_lengths[index_value];
  }

  // index_transition (src/basis/mod.rs:1561-1580)
  bool index_transition(u128 state, size_t source_orbit_size, size_t* row, C64* amplitude) const {
    if (!symmetric()) {
      if (!index(state, row)) return false;
      *amplitude = C64(1.0, 0.0);
      return true;
    }
    auto it = lookup.find(state);
    if (it == lookup.end()) return false;
    if (!index(it->second.representative, row)) fail(ERR_STATE_NOT_IN_BASIS, "");
    double scale = std::sqrt(static_cast<double>(source_orbit_size) /
                             static_cast<double>(it->second.orbit_size));
    *amplitude = scale * std::conj(it->second.phase);
    return true;
  }

  // visit_unreduced_local_transitions_with_symbols (src/basis/mod.rs:1122-1232)
  template <typename Visit>
  void visit_transitions(u128 state, const std::vector<char>& symbols,
                         const std::vector<size_t>& coupling_sites, Visit&& visit) const {
    if (symbols.size() != coupling_sites.size())
      fail(ERR_INVALID_COUPLING, "operator arity " + std::to_string(symbols.size()) +
                                     " does not match " + std::to_string(coupling_sites.size()) + " sites");
    struct Pending { u128 encoded; C64 amplitude; size_t remaining; };
    std::vector<Pending> pending;
    pending.push_back({state, C64(1.0, 0.0), symbols.size()});
    while (!pending.empty()) {
      Pending item = pending.back();
      pending.pop_back();
      u128 encoded = item.encoded;
      C64 amplitude = item.amplitude;
      size_t remaining = item.remaining;
      for (;;) {
        if (remaining == 0) {
          visit(encoded, amplitude);
          break;
        }
        size_t position = remaining - 1;
        size_t site = coupling_sites[position];
        char op = symbols[position];
        if (site >= sites)
          fail(ERR_INVALID_SITE, "site " + std::to_string(site) + " is outside a lattice with " +
                                     std::to_string(sites) + " sites");
        u128 place = static_cast<u128>(1) << site;
        int digit = static_cast<int>((encoded >> site) & 1);
        double raise_factor = raise_factors[digit];
        double lower_factor = lower_factors[digit];
        bool dead = false;
        switch (op) {
          case 'I': break;
          case 'z': {
            double factor = z_factors[digit];
            if (factor == 0.0) { dead = true; break; }
            amplitude *= factor;
            break;
          }
          case '+':
            if (raise_factor == 0.0) { dead = true; break; }
            encoded += place;
            if (raise_factor != 1.0) amplitude *= raise_factor;
            break;
          case '-':
            if (lower_factor == 0.0) { dead = true; break; }
            encoded -= place;
            if (lower_factor != 1.0) amplitude *= lower_factor;
            break;
          case 'x':
          case 'y': {
            double scale = normalization == 2 ? 1.0 : 0.5;
            C64 raise_phase = op == 'x' ? C64(scale, 0.0) : C64(0.0, -scale);
            C64 lower_phase = op == 'x' ? C64(scale, 0.0) : C64(0.0, scale);
            bool can_raise = raise_factor != 0.0, can_lower = lower_factor != 0.0;
            if (can_raise && can_lower) {
              pending.push_back({encoded - place, amplitude * (lower_phase * lower_factor), position});
              encoded += place;
              amplitude *= raise_phase * raise_factor;
            } else if (can_raise) {
              encoded += place;
              amplitude *= raise_phase * raise_factor;
            } else if (can_lower) {
              encoded -= place;
              amplitude *= lower_phase * lower_factor;
            } else {
              dead = true;
            }
            break;
          }
          default:
            fail(ERR_INVALID_OPERATOR, std::string(1, op));
        }
        if (dead) break;
        remaining = position;
      }
    }
  }
};

// The per-orbit part of spin_symmetry_sector (src/basis/mod.rs:790-841):
// projection coefficients of the orbit of `representative` (its minimum),
// the drop of |c| <= 1e-12, the gauge by the representative's coefficient,
// the normalisation check and the SymmetryImage of every member. Returns
// false when the projection vanishes (the orbit is not in the sector).
template <typename Lookup>
bool project_orbit(u128 representative, size_t sites, size_t translations, long normalized, int parity,
                   bool has_momentum, Lookup& lookup, size_t* orbit_size_out) {
  std::unordered_map<u128, C64, U128Hash> coefficients;
  for (size_t shift = 0; shift < translations; ++shift) {
    double angle = has_momentum ? -(2.0 * M_PI) * static_cast<double>(normalized * shift) /
                                      static_cast<double>(sites)
                                : 0.0;
    C64 character = std::polar(1.0, angle);
    u128 translated = rotate_lattice_state(representative, shift, sites);
    coefficients[translated] += character;
    if (parity != 0) {
      u128 reflected = reflect_lattice_state(translated, sites);
      coefficients[reflected] += static_cast<double>(parity) * character;
    }
  }
  for (auto it = coefficients.begin(); it != coefficients.end();) {
    if (std::abs(it->second) > 1.0e-12) ++it; else it = coefficients.erase(it);
  }
  if (coefficients.empty()) return false;
  auto rep_it = coefficients.find(representative);
  if (rep_it == coefficients.end())
    fail(ERR_INCOMPATIBLE_SYMMETRY, "symmetry projection removed its orbit representative");
  C64 representative_coefficient = rep_it->second;
  C64 gauge = representative_coefficient / std::abs(representative_coefficient);
  double norm_sq = 0.0;
  for (auto& entry : coefficients) norm_sq += std::norm(entry.second);
  double norm = std::sqrt(norm_sq);
  size_t orbit_size = coefficients.size();
  double expected = 1.0 / std::sqrt(static_cast<double>(orbit_size));
  for (auto& entry : coefficients) {
    C64 normalized_value = entry.second / (gauge * norm);
    if (std::abs(std::abs(normalized_value) - expected) > 1.0e-10)
      fail(ERR_INCOMPATIBLE_SYMMETRY,
           "symmetry projection does not define a one-dimensional orbit sector");
    lookup[entry.first] = {representative, normalized_value / expected, orbit_size};
  }
  *orbit_size_out = orbit_size;
  return true;
}

// spin_symmetry_sector (src/basis/mod.rs:715-848)
void spin_symmetry_sector(SpinBasis& basis, std::vector<u128> parent_states, bool has_momentum,
                          long momentum, int parity) {
  size_t sites = basis.sites;
  if (sites == 0) fail(ERR_INVALID_SECTOR, "symmetry sectors require at least one site");
  if (parity != 0 && parity != -1 && parity != 1)
    fail(ERR_INVALID_SECTOR, "parity must be either -1 or +1");
  long normalized = 0;
  if (has_momentum) {
    long L = static_cast<long>(sites);
    normalized = ((momentum % L) + L) % L;
  }
  if (parity != 0 && has_momentum && normalized != 0 && 2 * normalized != static_cast<long>(sites))
    fail(ERR_INCOMPATIBLE_SYMMETRY,
         "parity can share a one-dimensional sector with momentum only at k=0 or k=pi");
  basis.has_momentum = has_momentum;
  basis.momentum = static_cast<size_t>(normalized);
  basis.parity = parity;

  if (!has_momentum && parity == 0) {
    basis.orbit_lengths.assign(parent_states.size(), 1);
    basis.states = std::move(parent_states);
    return;  // the no-symmetry lookup is the identity and is never consulted
  }

  std::unordered_set<u128, U128Hash> parent_lookup(parent_states.begin(), parent_states.end());
  size_t translations = has_momentum ? sites : 1;
  std::unordered_set<u128, U128Hash> visited;
  visited.reserve(parent_states.size());
  std::vector<std::pair<u128, size_t>> sectors;
  basis.lookup.reserve(parent_states.size());

  for (u128 seed : parent_states) {
    if (visited.count(seed)) continue;
    std::unordered_set<u128, U128Hash> orbit;
    for (size_t shift = 0; shift < translations; ++shift) {
      u128 translated = rotate_lattice_state(seed, shift, sites);
      orbit.insert(translated);
      if (parity != 0) orbit.insert(reflect_lattice_state(translated, sites));
    }
    for (u128 s : orbit)
      if (!parent_lookup.count(s))
        fail(ERR_INCOMPATIBLE_SYMMETRY, "symmetry map leaves the selected magnetization sector");
    visited.insert(orbit.begin(), orbit.end());
    u128 representative = *std::min_element(orbit.begin(), orbit.end());
    size_t orbit_size = 0;
    if (!project_orbit(representative, sites, translations, normalized, parity, has_momentum, basis.lookup,
                       &orbit_size))
      continue;
    sectors.push_back({representative, orbit_size});
  }
  std::sort(sectors.begin(), sectors.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });
  basis.states.resize(sectors.size());
  basis.orbit_lengths.resize(sectors.size());
  for (size_t i = 0; i < sectors.size(); ++i) {
    basis.states[i] = sectors[i].first;
    basis.orbit_lengths[i] = sectors[i].second;
  }
}

// SpinBasisBuilder::build for spin one half (src/basis/mod.rs:1312-1412)
std::unique_ptr<SpinBasis> build_spin_basis(size_t sites, long up, bool has_momentum, long momentum,
                                            int parity, int normalization) {
  auto basis = std::make_unique<SpinBasis>();
  basis->sites = sites;
  basis->up = up;
  basis->normalization = normalization;
  const double spin = 0.5;
  for (int digit = 0; digit < 2; ++digit) {
    double magnetic = digit - spin;
    basis->z_factors[digit] = normalization == 0 ? magnetic : 2.0 * magnetic;
    double ladder_scale = normalization == 1 ? 2.0 : 1.0;
    basis->raise_factors[digit] =
        (digit + 1 < 2 ? std::sqrt(spin * (spin + 1.0) - magnetic * (magnetic + 1.0)) : 0.0) * ladder_scale;
    basis->lower_factors[digit] =
        (digit > 0 ? std::sqrt(spin * (spin + 1.0) - magnetic * (magnetic - 1.0)) : 0.0) * ladder_scale;
  }
  std::vector<u128> parent = fixed_weight_states(sites, up);
  spin_symmetry_sector(*basis, std::move(parent), has_momentum, momentum, parity);
  return basis;
}

// ----------------------------------------------------------------------------
// Operator terms and assembly (src/operator/mod.rs:51-319, 2002-2216)
// ----------------------------------------------------------------------------
struct Coupling {
  C64 coefficient;
  std::vector<size_t> sites;
};
struct Term {
  std::vector<char> symbols;
  std::string label;
  std::vector<Coupling> couplings;
};

// Operator stored as row-sorted triplets (the MatrixFree/CSR order of
// src/operator/mod.rs:2172-2176). All storage formats give the same action.
struct Operator {
  size_t rows = 0, cols = 0;
  std::vector<size_t> row_ptr;
  std::vector<size_t> col_idx;
  std::vector<C64> values;
  bool real = true;

  C64 value_at(size_t row, size_t col) const {
    auto begin = col_idx.begin() + static_cast<long>(row_ptr[row]);
    auto end = col_idx.begin() + static_cast<long>(row_ptr[row + 1]);
    auto it = std::lower_bound(begin, end, col);
    if (it != end && *it == col) return values[static_cast<size_t>(it - col_idx.begin())];
    return C64(0.0, 0.0);
  }

  // is_hermitian (src/operator/mod.rs:1313-1398, entry_is_hermitian 1233-1242)
  bool is_hermitian(double tolerance) const {
    if (rows != cols) return false;
    for (size_t r = 0; r < rows; ++r)
      for (size_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p)
        if (std::abs(values[p] - std::conj(value_at(col_idx[p], r))) > tolerance) return false;
    return true;
  }

  // apply / apply_real_coefficients (src/operator/mod.rs:1487-1548, 1244-1311)
  void apply(const C64* input, C64* output) const {
    for (size_t r = 0; r < rows; ++r) {
      C64 acc(0.0, 0.0);
      if (real) {
        for (size_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
          double coefficient = values[p].real();
          acc += C64(coefficient * input[col_idx[p]].real(), coefficient * input[col_idx[p]].imag());
        }
      } else {
        for (size_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) acc += values[p] * input[col_idx[p]];
      }
      output[r] = acc;
    }
  }

  // apply_real (src/operator/mod.rs:1414-1485)
  void apply_real(const double* input, double* output) const {
    if (!real) fail(ERR_UNSUPPORTED_BACKEND, "real action requires an operator with real-valued storage");
    for (size_t r = 0; r < rows; ++r) {
      double acc = 0.0;
      for (size_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) acc += values[p].real() * input[col_idx[p]];
      output[r] = acc;
    }
  }
};

// operator_number_changes (src/basis/mod.rs:294-325)
std::vector<int> operator_number_changes(const std::string& op) {
  std::vector<int> changes{0};
  for (char c : op) {
    if (c == '|') continue;
    switch (c) {
      case '+': for (int& v : changes) v += 1; break;
      case '-': for (int& v : changes) v -= 1; break;
      case 'x':
      case 'y': {
        std::vector<int> lowered = changes;
        for (int& v : changes) v += 1;
        for (int& v : lowered) v -= 1;
        changes.insert(changes.end(), lowered.begin(), lowered.end());
        std::sort(changes.begin(), changes.end());
        changes.erase(std::unique(changes.begin(), changes.end()), changes.end());
        break;
      }
      case 'I': case 'n': case 'z': break;
      default: fail(ERR_INVALID_OPERATOR, op);
    }
  }
  return changes;
}

// selected_sectors_preserve_changes for a single fixed sector (src/basis/mod.rs:348-371)
bool basis_preserves(const SpinBasis& basis, const std::string& op) {
  std::vector<int> changes = operator_number_changes(op);
  if (basis.up < 0) return true;
  long fixed = basis.up;
  long maximum = static_cast<long>(basis.sites);
  for (int change : changes) {
    long target = fixed + change;
    if (!(target < 0 || target > maximum || target == fixed)) return false;
  }
  return true;
}

// operator_sum_preserves_particle_sector (src/operator/mod.rs:1963-2033)
bool operator_sum_preserves_particle_sector(const SpinBasis& basis, const std::vector<Term>& terms) {
  std::map<std::tuple<size_t, std::string, std::vector<size_t>>, C64> components;
  for (const Term& term : terms) {
    for (const Coupling& coupling : term.couplings) {
      std::vector<std::tuple<size_t, std::string, C64>> expanded{{0, std::string(), C64(1.0, 0.0)}};
      for (char symbol : term.label) {
        if (symbol == 'x' || symbol == 'y') {
          std::vector<std::tuple<size_t, std::string, C64>> next;
          for (auto& [degree, prefix, coefficient] : expanded) {
            C64 raise_phase = symbol == 'x' ? C64(1.0, 0.0) : C64(0.0, -1.0);
            C64 lower_phase = symbol == 'x' ? C64(1.0, 0.0) : C64(0.0, 1.0);
            next.push_back({degree + 1, prefix + '+', coefficient * raise_phase});
            next.push_back({degree + 1, prefix + '-', coefficient * lower_phase});
          }
          expanded = std::move(next);
        } else if (symbol == 'I' || symbol == 'n' || symbol == 'z' || symbol == '+' || symbol == '-' || symbol == '|') {
          for (auto& item : expanded) std::get<1>(item).push_back(symbol);
        } else {
          fail(ERR_INVALID_OPERATOR, term.label);
        }
      }
      for (auto& [degree, op, coefficient] : expanded)
        components[{degree, op, coupling.sites}] += coupling.coefficient * coefficient;
    }
  }
  for (auto& [key, coefficient] : components)
    if (std::abs(coefficient) > EPS && !basis_preserves(basis, std::get<1>(key))) return false;
  return true;
}

// OperatorBuilder::build (src/operator/mod.rs:2091-2216), square case.
std::unique_ptr<Operator> build_operator(const SpinBasis& basis, const std::vector<Term>& terms,
                                         bool check_hermitian, bool check_particles) {
  for (const Term& term : terms)
    for (const Coupling& coupling : term.couplings) {
      if (coupling.sites.size() != term.symbols.size())
        fail(ERR_INVALID_COUPLING, "operator \"" + term.label + "\" has arity " +
                                       std::to_string(term.symbols.size()) + ", but a coupling has " +
                                       std::to_string(coupling.sites.size()) + " sites");
      if (!std::isfinite(coupling.coefficient.real()) || !std::isfinite(coupling.coefficient.imag()))
        fail(ERR_INVALID_COUPLING, "coupling coefficients must be finite");
    }
  if (check_particles && !operator_sum_preserves_particle_sector(basis, terms))
    fail(ERR_INVALID_SECTOR, "operator sum does not preserve the selected particle sector");
  size_t dimension = basis.len();
  struct Triplet { size_t row, col; C64 value; };
  std::vector<Triplet> entries;
  std::vector<std::pair<size_t, C64>> column_entries;
  for (size_t column = 0; column < dimension; ++column) {
    column_entries.clear();
    u128 source_state = basis.states[column];
    size_t source_orbit = basis.transition_orbit_size(source_state);
    for (const Term& term : terms)
      for (const Coupling& coupling : term.couplings)
        basis.visit_transitions(source_state, term.symbols, coupling.sites, [&](u128 target, C64 amp) {
          size_t row;
          C64 reduction;
          if (!basis.index_transition(target, source_orbit, &row, &reduction)) return;
          column_entries.push_back({row, coupling.coefficient * amp * reduction});
        });
    std::stable_sort(column_entries.begin(), column_entries.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    size_t position = 0;
    while (position < column_entries.size()) {
      size_t row = column_entries[position].first;
      C64 value = column_entries[position].second;
      ++position;
      while (position < column_entries.size() && column_entries[position].first == row) {
        value += column_entries[position].second;
        ++position;
      }
      if (std::abs(value) <= EPS) continue;
      entries.push_back({row, column, value});
    }
  }
  std::stable_sort(entries.begin(), entries.end(), [](const Triplet& a, const Triplet& b) {
    return a.row != b.row ? a.row < b.row : a.col < b.col;
  });
  auto op = std::make_unique<Operator>();
  op->rows = op->cols = dimension;
  op->row_ptr.assign(dimension + 1, 0);
  op->col_idx.resize(entries.size());
  op->values.resize(entries.size());
  for (size_t i = 0; i < entries.size(); ++i) {
    op->row_ptr[entries[i].row + 1] += 1;
    op->col_idx[i] = entries[i].col;
    op->values[i] = entries[i].value;
    if (entries[i].value.imag() != 0.0) op->real = false;
  }
  for (size_t r = 0; r < dimension; ++r) op->row_ptr[r + 1] += op->row_ptr[r];
  if (check_hermitian && !op->is_hermitian(1.0e-12)) fail(ERR_NON_HERMITIAN, "");
  return op;
}

// Operator::from_triplets (src/operator/mod.rs:755-816): duplicates summed,
// |v| <= eps dropped, row-major order.
std::unique_ptr<Operator> operator_from_triplets(size_t n, const std::vector<size_t>& rows,
                                                 const std::vector<size_t>& cols,
                                                 const std::vector<C64>& vals) {
  std::map<std::pair<size_t, size_t>, C64> accumulated;
  for (size_t i = 0; i < rows.size(); ++i) {
    if (rows[i] >= n || cols[i] >= n || !std::isfinite(vals[i].real()) || !std::isfinite(vals[i].imag()))
      fail(ERR_INVALID_COUPLING, "triplet index is out of bounds or its value is non-finite");
    accumulated[{rows[i], cols[i]}] += vals[i];
  }
  auto op = std::make_unique<Operator>();
  op->rows = op->cols = n;
  op->row_ptr.assign(n + 1, 0);
  for (auto& [key, value] : accumulated) {
    if (std::abs(value) <= EPS) continue;
    op->row_ptr[key.first + 1] += 1;
    op->col_idx.push_back(key.second);
    op->values.push_back(value);
    if (value.imag() != 0.0) op->real = false;
  }
  for (size_t r = 0; r < n; ++r) op->row_ptr[r + 1] += op->row_ptr[r];
  return op;
}

// ----------------------------------------------------------------------------
// Dense symmetric / Hermitian eigensolvers (stand-in for nalgebra/faer).
// ----------------------------------------------------------------------------

// Symmetric tridiagonal eigenproblem by implicit QL with Wilkinson shifts
// (Bowdler, Martin, Reinsch & Wilkinson, "The QR and QL algorithms for
// symmetric matrices", Numer. Math. 11 (1968)). Eigenvector matrix is
// column-major: z[row + n*col].
void tridiagonal_eigen(size_t n, std::vector<double> d, std::vector<double> e, std::vector<double>& values,
                       std::vector<double>& z) {
  z.assign(n * n, 0.0);
  for (size_t i = 0; i < n; ++i) z[i + n * i] = 1.0;
  e.resize(n, 0.0);
  for (size_t l = 0; l < n; ++l) {
    int iterations = 0;
    for (;;) {
      size_t m = l;
      for (; m + 1 < n; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= EPS * dd) break;
      }
      if (m == l) break;
      if (++iterations > 60) fail(ERR_INTERNAL_STATE, "tridiagonal eigensolver did not converge");
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
      double s = 1.0, c = 1.0, p = 0.0;
      size_t i = m;
      bool underflow = false;
      while (i-- > l) {
        double f = s * e[i];
        double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (size_t k = 0; k < n; ++k) {
          f = z[k + n * (i + 1)];
          z[k + n * (i + 1)] = s * z[k + n * i] + c * f;
          z[k + n * i] = c * z[k + n * i] - s * f;
        }
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  values = d;
}

// Cyclic Jacobi for a dense Hermitian matrix (row-major a[i*n+j]). Returns the
// eigenvalues (unsorted) and column-major eigenvectors v[row + n*col].
void hermitian_jacobi(size_t n, std::vector<C64> a, std::vector<double>& values, std::vector<C64>& v) {
  v.assign(n * n, C64(0.0, 0.0));
  for (size_t i = 0; i < n; ++i) v[i + n * i] = C64(1.0, 0.0);
  auto A = [&](size_t i, size_t j) -> C64& { return a[i * n + j]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, total = 0.0;
    for (size_t i = 0; i < n; ++i)
      for (size_t j = 0; j < n; ++j) {
        total += std::norm(A(i, j));
        if (i != j) off += std::norm(A(i, j));
      }
    if (off <= 1e-30 * std::max(total, 1e-300) || off == 0.0) break;
    for (size_t p = 0; p + 1 < n; ++p)
      for (size_t q = p + 1; q < n; ++q) {
        C64 apq = A(p, q);
        double magnitude = std::abs(apq);
        if (magnitude == 0.0) continue;
        double app = A(p, p).real(), aqq = A(q, q).real();
        // Rotation that annihilates |a_pq| after removing its phase.
        C64 phase = apq / magnitude;
        double theta = (aqq - app) / (2.0 * magnitude);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0);
        double s = t * c;
        // Columns: A <- A J, with J = [[c, s*phase],[-s*conj(phase), c]] on (p,q).
        for (size_t k = 0; k < n; ++k) {
          C64 akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * std::conj(phase) * akq;
          A(k, q) = s * phase * akp + c * akq;
        }
        for (size_t k = 0; k < n; ++k) {
          C64 apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * phase * aqk;
          A(q, k) = s * std::conj(phase) * apk + c * aqk;
        }
        A(p, q) = C64(0.0, 0.0);
        A(q, p) = C64(0.0, 0.0);
        A(p, p) = C64(A(p, p).real(), 0.0);
        A(q, q) = C64(A(q, q).real(), 0.0);
        for (size_t k = 0; k < n; ++k) {
          C64 vkp = v[k + n * p], vkq = v[k + n * q];
          v[k + n * p] = c * vkp - s * std::conj(phase) * vkq;
          v[k + n * q] = s * phase * vkp + c * vkq;
        }
      }
  }
  values.resize(n);
  for (size_t i = 0; i < n; ++i) values[i] = A(i, i).real();
}

// ----------------------------------------------------------------------------
// Eigensolvers (src/solve/mod.rs:349-2452)
// ----------------------------------------------------------------------------
enum Target { SA = 0, LA = 1, SM = 2, LM = 3, BE = 4, SHIFT = 5 };

struct EigshOptions {
  size_t eigenpairs = 1;
  int target = SA;
  double shift = 0.0;
  size_t krylov_dimension = 0;  // 0 = None
  double tolerance = 1.0e-10;
  size_t max_iterations = 1000;
  uint64_t seed = 0;
};

struct Eigensystem {
  std::vector<double> eigenvalues;
  std::vector<std::vector<C64>> eigenvectors;
  std::vector<double> residuals;
  size_t iterations = 0;
  size_t reorthogonalization_passes = 0;
  size_t conditional_second_passes = 0;
};

constexpr size_t GUARANTEED_DENSE_EIGSH_CROSSOVER = 128;
constexpr size_t AUTOMATIC_DENSE_EIGSH_CROSSOVER = 256;
constexpr size_t FULL_KRYLOV_DENSE_FALLBACK = 2048;
constexpr size_t TRIDIAGONAL_LANCZOS_WINDOW = 96;
const double DGKS_THRESHOLD = 1.0 / std::sqrt(2.0);

bool use_dense_eigsh(size_t dimension, const EigshOptions& o) {
  return dimension <= GUARANTEED_DENSE_EIGSH_CROSSOVER ||
         (dimension <= AUTOMATIC_DENSE_EIGSH_CROSSOVER && o.krylov_dimension == 0);
}

// EigshOptions::validate (src/solve/mod.rs:425-448)
void validate_options(const EigshOptions& o, size_t dimension) {
  if (o.eigenpairs == 0 || o.eigenpairs >= dimension)
    fail(ERR_INVALID_OPTIONS, "eigenpairs must be positive and smaller than the operator dimension");
  if (!std::isfinite(o.tolerance) || o.tolerance <= 0.0 || o.max_iterations == 0)
    fail(ERR_INVALID_OPTIONS, "tolerance and max_iterations must be positive");
  if (o.krylov_dimension != 0 && (o.krylov_dimension <= o.eigenpairs || o.krylov_dimension > dimension))
    fail(ERR_INVALID_OPTIONS, "krylov_dimension must exceed eigenpairs and not exceed dimension");
  if (o.target == SHIFT && !std::isfinite(o.shift)) fail(ERR_INVALID_OPTIONS, "shift must be finite");
  if (o.target == SHIFT)
    fail(ERR_UNSUPPORTED_BACKEND, "shift-invert eigsh targets are outside this engine");
}

// Scalar helpers shared by the real and complex Lanczos restatements.
inline double conj_s(double v) { return v; }
inline C64 conj_s(C64 v) { return std::conj(v); }
inline double norm_sq_s(double v) { return v * v; }
inline double norm_sq_s(C64 v) { return std::norm(v); }
inline double real_s(double v) { return v; }
inline double real_s(C64 v) { return v.real(); }

template <typename T>
T inner(const std::vector<T>& a, const std::vector<T>& b) {
  T sum = T(0);
  for (size_t i = 0; i < a.size(); ++i) sum += conj_s(a[i]) * b[i];
  return sum;
}
template <typename T>
double vnorm(const std::vector<T>& v) {
  double s = 0.0;
  for (auto& x : v) s += norm_sq_s(x);
  return std::sqrt(s);
}

template <typename T>
void apply_op(const Operator& op, const std::vector<T>& x, std::vector<T>& y);
template <>
void apply_op<double>(const Operator& op, const std::vector<double>& x, std::vector<double>& y) {
  op.apply_real(x.data(), y.data());
}
template <>
void apply_op<C64>(const Operator& op, const std::vector<C64>& x, std::vector<C64>& y) {
  op.apply(x.data(), y.data());
}

// normalize / normalize_real (src/solve/mod.rs:690-706, 1101-1113)
template <typename T>
void normalize_vec(std::vector<T>& v) {
  double n = vnorm(v);
  if (!std::isfinite(n) || n <= EPS) fail_nonconvergence(0, n);
  for (auto& x : v) x /= n;
}

// deterministic_start (src/solve/mod.rs:729-742)
std::vector<C64> deterministic_start(size_t dimension, uint64_t seed) {
  uint64_t state = seed | 1;
  std::vector<C64> v(dimension);
  for (size_t i = 0; i < dimension; ++i) {
    state = state * 6364136223846793005ULL + 1442695040888963407ULL;
    uint64_t mantissa = state >> 11;
    double value = static_cast<double>(mantissa) / static_cast<double>(1ULL << 53) - 0.5;
    v[i] = C64(value, 0.0);
  }
  normalize_vec(v);
  return v;
}

template <typename T>
std::vector<T> from_complex(const std::vector<C64>& v);
template <>
std::vector<double> from_complex<double>(const std::vector<C64>& v) {
  std::vector<double> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) r[i] = v[i].real();
  return r;
}
template <>
std::vector<C64> from_complex<C64>(const std::vector<C64>& v) { return v; }

std::vector<C64> to_complex(const std::vector<double>& v) {
  std::vector<C64> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) r[i] = C64(v[i], 0.0);
  return r;
}
std::vector<C64> to_complex(const std::vector<C64>& v) { return v; }

// select_indices (src/solve/mod.rs:1002-1036)
std::vector<size_t> select_indices(const std::vector<double>& values, int target, size_t count) {
  std::vector<size_t> idx(values.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
  if (target == BE) {
    std::sort(idx.begin(), idx.end(), [&](size_t l, size_t r) {
      return values[l] != values[r] ? values[l] < values[r] : l < r;
    });
    size_t lower = count / 2, upper = count - lower;
    std::vector<size_t> selected(idx.begin(), idx.begin() + static_cast<long>(std::min(lower, idx.size())));
    for (size_t i = 0; i < upper && i < idx.size(); ++i) selected.push_back(idx[idx.size() - 1 - i]);
    std::stable_sort(selected.begin(), selected.end(), [&](size_t l, size_t r) { return values[l] < values[r]; });
    return selected;
  }
  auto key_less = [&](size_t l, size_t r) {
    double a = values[l], b = values[r];
    int ord = 0;
    switch (target) {
      case SA: ord = a < b ? -1 : (a > b ? 1 : 0); break;
      case LA: ord = b < a ? -1 : (b > a ? 1 : 0); break;
      case SM: ord = std::fabs(a) < std::fabs(b) ? -1 : (std::fabs(a) > std::fabs(b) ? 1 : 0); break;
      case LM: ord = std::fabs(b) < std::fabs(a) ? -1 : (std::fabs(b) > std::fabs(a) ? 1 : 0); break;
      default: break;
    }
    return ord != 0 ? ord < 0 : l < r;
  };
  std::sort(idx.begin(), idx.end(), key_less);
  if (idx.size() > count) idx.resize(count);
  return idx;
}

bool candidate_before(double a, double b, int target) {
  switch (target) {
    case SA: case BE: return a < b;
    case LA: return b < a;
    case SM: return std::fabs(a) < std::fabs(b);
    case LM: return std::fabs(b) < std::fabs(a);
    default: return a < b;
  }
}

// dgks_reorthogonalize_real/_complex (src/solve/mod.rs:1050-1099)
template <typename T>
std::pair<double, bool> dgks_reorthogonalize(const std::vector<std::vector<T>>& basis, std::vector<T>& out) {
  double before = vnorm(out);
  for (auto& b : basis) {
    T overlap = inner(b, out);
    for (size_t i = 0; i < out.size(); ++i) out[i] -= overlap * b[i];
  }
  double after = vnorm(out);
  if (before > EPS && after <= DGKS_THRESHOLD * before) {
    for (auto& b : basis) {
      T overlap = inner(b, out);
      for (size_t i = 0; i < out.size(); ++i) out[i] -= overlap * b[i];
    }
    return {vnorm(out), true};
  }
  return {after, false};
}

// lanczos_eigsh_real (src/solve/mod.rs:1116-1282) / lanczos_eigsh complex (1285-1456)
template <typename T>
Eigensystem lanczos_eigsh_t(const Operator& op, const EigshOptions& options, const std::vector<C64>* initial) {
  size_t dimension = op.rows;
  size_t requested = options.krylov_dimension ? options.krylov_dimension
                                               : std::max<size_t>(8 * options.eigenpairs + 64, 256);
  size_t krylov = std::min({requested, options.max_iterations, dimension});
  if (krylov <= options.eigenpairs)
    fail(ERR_INVALID_OPTIONS, "the effective Krylov dimension must exceed eigenpairs");
  std::vector<T> first;
  if (initial) {
    if (initial->size() != dimension) fail(ERR_DIMENSION_MISMATCH, "eigsh initial vector does not match the operator");
    first = from_complex<T>(*initial);
    normalize_vec(first);
  } else {
    first = from_complex<T>(deterministic_start(dimension, options.seed));
  }
  std::vector<std::vector<T>> basis;
  basis.push_back(first);
  std::vector<double> alphas, betas;
  std::vector<T> output(dimension);
  size_t passes = 0, second_passes = 0;
  for (size_t iteration = 0; iteration < krylov; ++iteration) {
    apply_op(op, basis[iteration], output);
    double alpha = real_s(inner(basis[iteration], output));
    alphas.push_back(alpha);
    for (size_t i = 0; i < dimension; ++i) output[i] -= alpha * basis[iteration][i];
    if (iteration > 0) {
      double beta = betas[iteration - 1];
      for (size_t i = 0; i < dimension; ++i) output[i] -= beta * basis[iteration - 1][i];
    }
    auto [beta, second] = dgks_reorthogonalize(basis, output);
    passes += 1 + (second ? 1 : 0);
    if (second) second_passes += 1;
    if (iteration + 1 == krylov || beta <= 1.0e-14) break;
    betas.push_back(beta);
    for (auto& v : output) v /= beta;
    basis.push_back(output);
  }
  if (basis.size() <= options.eigenpairs) fail_nonconvergence(basis.size(), INFINITY);
  size_t size = basis.size();
  std::vector<double> d(alphas.begin(), alphas.begin() + static_cast<long>(size));
  std::vector<double> e(size, 0.0);
  for (size_t i = 0; i + 1 < size; ++i) e[i] = betas[i];
  std::vector<double> values, z;
  tridiagonal_eigen(size, d, e, values, z);
  std::vector<size_t> indices = select_indices(values, options.target, options.eigenpairs);
  struct Cand { double value; std::vector<T> vector; double residual; };
  std::vector<Cand> candidates;
  for (size_t index : indices) {
    std::vector<T> vector(dimension, T(0));
    for (size_t j = 0; j < size; ++j) {
      double coefficient = z[j + size * index];
      for (size_t i = 0; i < dimension; ++i) vector[i] += coefficient * basis[j][i];
    }
    normalize_vec(vector);
    apply_op(op, vector, output);
    double eigenvalue = real_s(inner(vector, output));
    double r = 0.0;
    for (size_t i = 0; i < dimension; ++i) r += norm_sq_s(output[i] - eigenvalue * vector[i]);
    candidates.push_back({eigenvalue, std::move(vector), std::sqrt(r)});
  }
  std::stable_sort(candidates.begin(), candidates.end(),
                   [&](const Cand& a, const Cand& b) { return candidate_before(a.value, b.value, options.target); });
  double failure = 0.0;
  for (auto& c : candidates)
    if (c.residual > options.tolerance * std::max(std::fabs(c.value), 1.0)) failure = std::max(failure, c.residual);
  if (failure > 0.0) fail_nonconvergence(size, failure);
  Eigensystem result;
  for (auto& c : candidates) {
    result.eigenvalues.push_back(c.value);
    result.residuals.push_back(c.residual);
    result.eigenvectors.push_back(to_complex(c.vector));
  }
  result.iterations = size;
  result.reorthogonalization_passes = passes;
  result.conditional_second_passes = second_passes;
  return result;
}

Eigensystem lanczos_eigsh(const Operator& op, const EigshOptions& options, const std::vector<C64>* initial) {
  bool real_compatible = op.real;
  if (initial)
    for (auto& v : *initial)
      if (std::fabs(v.imag()) > 1.0e-14) real_compatible = false;
  if (real_compatible) return lanczos_eigsh_t<double>(op, options, initial);
  return lanczos_eigsh_t<C64>(op, options, initial);
}

// orthonormalize_{real,complex}_with_projection (src/solve/mod.rs:1520-1575, 1587-1642)
template <typename T>
struct RitzCand {
  double value;
  std::vector<T> vector;
  double residual;
  std::vector<T> action;
};

template <typename T>
struct OrthoResult {
  bool ok;
  std::vector<T> vector;
  size_t passes, second_passes;
  std::vector<T> projection;
};

template <typename T>
OrthoResult<T> orthonormalize_with_projection(const std::vector<RitzCand<T>>& locked,
                                              const std::vector<std::vector<T>>& basis, std::vector<T> vector) {
  double before = vnorm(vector);
  for (auto& c : locked) {
    T overlap = inner(c.vector, vector);
    for (size_t i = 0; i < vector.size(); ++i) vector[i] -= overlap * c.vector[i];
  }
  std::vector<T> projection;
  for (auto& b : basis) {
    T overlap = inner(b, vector);
    projection.push_back(overlap);
    for (size_t i = 0; i < vector.size(); ++i) vector[i] -= overlap * b[i];
  }
  double norm = vnorm(vector);
  bool second = before > EPS && norm <= DGKS_THRESHOLD * before;
  if (second) {
    for (auto& c : locked) {
      T overlap = inner(c.vector, vector);
      for (size_t i = 0; i < vector.size(); ++i) vector[i] -= overlap * c.vector[i];
    }
    for (auto& b : basis) {
      T overlap = inner(b, vector);
      for (size_t i = 0; i < vector.size(); ++i) vector[i] -= overlap * b[i];
    }
    norm = vnorm(vector);
  }
  size_t passes = 1 + (second ? 1 : 0), seconds = second ? 1 : 0;
  if (!std::isfinite(norm) || norm <= 1.0e-14) return {false, {}, passes, seconds, projection};
  for (auto& v : vector) v /= norm;
  return {true, std::move(vector), passes, seconds, projection};
}

// thick_restart_dimension (src/solve/mod.rs:1644-1649)
size_t thick_restart_dimension(const EigshOptions& o, size_t dimension) {
  size_t window = o.krylov_dimension ? o.krylov_dimension : std::max<size_t>(4 * o.eigenpairs + 24, 32);
  return std::min(window, dimension);
}

// Projected (small) Hermitian eigenproblem; values ascending is not required.
void projected_eigen(size_t size, const std::vector<std::vector<double>>& columns, std::vector<double>& values,
                     std::vector<double>& vectors_cm) {
  std::vector<C64> a(size * size, C64(0.0, 0.0));
  for (size_t col = 0; col < size; ++col)
    for (size_t row = 0; row <= col && row < columns[col].size(); ++row) {
      a[row * size + col] = C64(columns[col][row], 0.0);
      a[col * size + row] = C64(columns[col][row], 0.0);
    }
  std::vector<C64> v;
  hermitian_jacobi(size, a, values, v);
  vectors_cm.resize(size * size);
  for (size_t i = 0; i < size * size; ++i) vectors_cm[i] = v[i].real();
}
void projected_eigen(size_t size, const std::vector<std::vector<C64>>& columns, std::vector<double>& values,
                     std::vector<C64>& vectors_cm) {
  std::vector<C64> a(size * size, C64(0.0, 0.0));
  for (size_t col = 0; col < size; ++col)
    for (size_t row = 0; row <= col && row < columns[col].size(); ++row) {
      a[row * size + col] = columns[col][row];
      a[col * size + row] = std::conj(columns[col][row]);
    }
  hermitian_jacobi(size, a, values, vectors_cm);
}

// thick_restarted_eigsh_real (src/solve/mod.rs:1651-1912) and complex (1914-2167)
template <typename T>
Eigensystem thick_restarted_eigsh_t(const Operator& op, const EigshOptions& options,
                                    const std::vector<std::vector<C64>>* initial_subspace) {
  size_t dimension = op.rows;
  size_t restart_dimension = thick_restart_dimension(options, dimension);
  if (restart_dimension <= options.eigenpairs)
    fail(ERR_INVALID_OPTIONS, "the effective Krylov dimension must exceed eigenpairs");
  struct Retained { std::vector<T> vector; bool has_action; std::vector<T> action; };
  std::vector<Retained> retained;
  if (initial_subspace)
    for (auto& v : *initial_subspace) retained.push_back({from_complex<T>(v), false, {}});
  std::vector<RitzCand<T>> locked;
  size_t iterations = 0, passes = 0, second_passes = 0;
  double last_residual = INFINITY;
  uint64_t cycle = 0;
  while (iterations < options.max_iterations && locked.size() < options.eigenpairs) {
    std::vector<std::vector<T>> basis, applied;
    bool reuse_actions = !retained.empty();
    for (auto& r : retained) reuse_actions = reuse_actions && r.has_action;
    for (auto& r : retained) {
      if (reuse_actions) {
        double norm = vnorm(r.vector);
        if (std::isfinite(norm) && norm > 1.0e-14) {
          for (auto& x : r.vector) x /= norm;
          for (auto& x : r.action) x /= norm;
          basis.push_back(std::move(r.vector));
          applied.push_back(std::move(r.action));
        }
      } else {
        auto o = orthonormalize_with_projection(locked, basis, std::move(r.vector));
        passes += o.passes;
        second_passes += o.second_passes;
        if (o.ok) basis.push_back(std::move(o.vector));
      }
      if (basis.size() >= restart_dimension / 2) break;
    }
    retained.clear();
    if (basis.empty()) {
      auto start = from_complex<T>(deterministic_start(dimension, options.seed + cycle * 0x9e3779b9ULL));
      auto o = orthonormalize_with_projection(locked, basis, std::move(start));
      passes += o.passes;
      second_passes += o.second_passes;
      if (o.ok) basis.push_back(std::move(o.vector));
    }
    if (basis.empty()) break;

    size_t known_actions = applied.size();
    std::vector<std::vector<T>> projection_columns;
    if (reuse_actions) {
      for (size_t column = 0; column < known_actions; ++column) {
        if (basis.size() >= restart_dimension) break;
        auto o = orthonormalize_with_projection(locked, basis, applied[column]);
        passes += o.passes;
        second_passes += o.second_passes;
        projection_columns.push_back(std::vector<T>(o.projection.begin(), o.projection.begin() + static_cast<long>(column + 1)));
        if (o.ok) basis.push_back(std::move(o.vector));
      }
    }
    size_t cursor = known_actions;
    while (cursor < basis.size() && iterations < options.max_iterations && applied.size() < restart_dimension) {
      std::vector<T> output(dimension);
      apply_op(op, basis[cursor], output);
      iterations += 1;
      applied.push_back(output);
      auto o = orthonormalize_with_projection(locked, basis, std::move(output));
      passes += o.passes;
      second_passes += o.second_passes;
      projection_columns.push_back(std::vector<T>(o.projection.begin(), o.projection.begin() + static_cast<long>(cursor + 1)));
      if (basis.size() < restart_dimension && o.ok) basis.push_back(std::move(o.vector));
      cursor += 1;
    }
    if (basis.size() > applied.size()) basis.resize(applied.size());
    if (basis.empty()) break;

    size_t size = basis.size();
    std::vector<double> values;
    std::vector<T> vecs;
    projected_eigen(size, projection_columns, values, vecs);
    size_t active_needed = options.eigenpairs - locked.size();
    size_t keep_limit = std::max<size_t>(std::min(active_needed, restart_dimension / 2), 1);
    std::vector<size_t> indices = select_indices(values, options.target, std::min(keep_limit, size));
    std::vector<RitzCand<T>> candidates;
    for (size_t index : indices) {
      std::vector<T> vector(dimension, T(0)), action(dimension, T(0));
      for (size_t j = 0; j < size; ++j) {
        T coefficient = vecs[j + size * index];
        for (size_t i = 0; i < dimension; ++i) vector[i] += coefficient * basis[j][i];
        for (size_t i = 0; i < dimension; ++i) action[i] += coefficient * applied[j][i];
      }
      double ritz_norm = vnorm(vector);
      if (!std::isfinite(ritz_norm) || ritz_norm <= EPS) fail_nonconvergence(iterations, ritz_norm);
      for (auto& x : vector) x /= ritz_norm;
      for (auto& x : action) x /= ritz_norm;
      double value = real_s(inner(vector, action));
      double r = 0.0;
      for (size_t i = 0; i < dimension; ++i) r += norm_sq_s(action[i] - value * vector[i]);
      candidates.push_back({value, std::move(vector), std::sqrt(r), std::move(action)});
    }
    std::stable_sort(candidates.begin(), candidates.end(), [&](const RitzCand<T>& a, const RitzCand<T>& b) {
      return candidate_before(a.value, b.value, options.target);
    });
    last_residual = 0.0;
    for (size_t i = 0; i < candidates.size() && i < active_needed; ++i)
      last_residual = std::max(last_residual, candidates[i].residual);
    std::vector<Retained> next_retained;
    for (size_t rank = 0; rank < candidates.size(); ++rank) {
      auto& c = candidates[rank];
      bool converged = c.residual <= options.tolerance * std::max(std::fabs(c.value), 1.0);
      if (rank < active_needed && converged && locked.size() < options.eigenpairs) {
        std::vector<std::vector<T>> empty;
        auto o = orthonormalize_with_projection(locked, empty, c.vector);
        passes += o.passes;
        second_passes += o.second_passes;
        if (o.ok) {
          RitzCand<T> l = c;
          l.vector = std::move(o.vector);
          locked.push_back(std::move(l));
        }
      } else if (next_retained.size() < keep_limit) {
        next_retained.push_back({std::move(c.vector), true, std::move(c.action)});
      }
    }
    retained = std::move(next_retained);
    cycle += 1;
  }
  if (locked.size() < options.eigenpairs) fail_nonconvergence(iterations, last_residual);
  std::stable_sort(locked.begin(), locked.end(), [&](const RitzCand<T>& a, const RitzCand<T>& b) {
    return candidate_before(a.value, b.value, options.target);
  });
  locked.resize(options.eigenpairs);
  Eigensystem result;
  for (auto& c : locked) {
    result.eigenvalues.push_back(c.value);
    result.residuals.push_back(c.residual);
    result.eigenvectors.push_back(to_complex(c.vector));
  }
  result.iterations = iterations;
  result.reorthogonalization_passes = passes;
  result.conditional_second_passes = second_passes;
  return result;
}

Eigensystem thick_restarted_eigsh(const Operator& op, const EigshOptions& options,
                                  const std::vector<std::vector<C64>>* initial_subspace) {
  bool real_compatible = op.real;
  if (initial_subspace)
    for (auto& v : *initial_subspace)
      for (auto& x : v)
        if (std::fabs(x.imag()) > 1.0e-14) real_compatible = false;
  if (real_compatible) return thick_restarted_eigsh_t<double>(op, options, initial_subspace);
  return thick_restarted_eigsh_t<C64>(op, options, initial_subspace);
}

// rayleigh_value_and_residual (src/solve/mod.rs:635-658)
std::pair<double, double> rayleigh(const Operator& op, const std::vector<C64>& v) {
  std::vector<C64> applied(v.size());
  op.apply(v.data(), applied.data());
  double norm_sq = real_s(inner(v, v));
  if (!std::isfinite(norm_sq) || norm_sq <= EPS) fail_nonconvergence(0, std::sqrt(norm_sq));
  double value = inner(v, applied).real() / norm_sq;
  double r = 0.0;
  for (size_t i = 0; i < v.size(); ++i) r += std::norm(applied[i] - value * v[i]);
  return {value, std::sqrt(r)};
}

// dense_eigsh (src/solve/mod.rs:2198-2240) via hermitian_eigenpairs_all (578-604)
Eigensystem dense_eigsh(const Operator& op, const EigshOptions& options) {
  size_t n = op.rows;
  std::vector<C64> dense(n * n, C64(0.0, 0.0));
  for (size_t r = 0; r < n; ++r)
    for (size_t p = op.row_ptr[r]; p < op.row_ptr[r + 1]; ++p) dense[r * n + op.col_idx[p]] += op.values[p];
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < n; ++c)
      if (std::abs(dense[r * n + c] - std::conj(dense[c * n + r])) > 1.0e-12) fail(ERR_NON_HERMITIAN, "");
  std::vector<double> values;
  std::vector<C64> vectors;
  hermitian_jacobi(n, dense, values, vectors);
  // faer returns ascending eigenvalues; keep that order before selection.
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return values[a] < values[b]; });
  std::vector<double> sorted(n);
  for (size_t i = 0; i < n; ++i) sorted[i] = values[order[i]];
  std::vector<size_t> indices = select_indices(sorted, options.target, options.eigenpairs);
  Eigensystem result;
  for (size_t index : indices) {
    std::vector<C64> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = vectors[i + n * order[index]];
    auto [value, residual] = rayleigh(op, v);
    result.eigenvalues.push_back(value);
    result.residuals.push_back(residual);
    result.eigenvectors.push_back(std::move(v));
  }
  result.iterations = 1;
  return result;
}

// expanding_lanczos_eigsh (src/solve/mod.rs:2242-2328)
Eigensystem expanding_lanczos_eigsh(const Operator& op, const EigshOptions& options,
                                    const std::vector<std::vector<C64>>* initial_subspace) {
  size_t dimension = op.rows;
  if (options.krylov_dimension == 0 && (!initial_subspace || initial_subspace->size() <= 1)) {
    const std::vector<C64>* initial = (initial_subspace && !initial_subspace->empty()) ? &(*initial_subspace)[0] : nullptr;
    size_t subspace = std::min({std::max<size_t>(8 * options.eigenpairs + 64, 256), dimension, options.max_iterations});
    size_t spent = 0;
    for (;;) {
      EigshOptions attempt = options;
      attempt.krylov_dimension = subspace;
      attempt.max_iterations = subspace;
      try {
        Eigensystem result = lanczos_eigsh(op, attempt, initial);
        result.iterations += spent;
        return result;
      } catch (const QError& error) {
        if (error.code != ERR_NON_CONVERGENCE) throw;
        spent += error.iterations;
        if (subspace == dimension && dimension <= FULL_KRYLOV_DENSE_FALLBACK) {
          Eigensystem result = dense_eigsh(op, options);
          result.iterations += spent;
          return result;
        }
        size_t remaining = options.max_iterations > spent ? options.max_iterations - spent : 0;
        size_t next = std::min({subspace * 2, dimension, remaining});
        if (next <= subspace) fail_nonconvergence(spent, error.residual);
        subspace = next;
      }
    }
  }
  if (options.krylov_dimension >= TRIDIAGONAL_LANCZOS_WINDOW && (!initial_subspace || initial_subspace->size() <= 1)) {
    const std::vector<C64>* initial = (initial_subspace && !initial_subspace->empty()) ? &(*initial_subspace)[0] : nullptr;
    return lanczos_eigsh(op, options, initial);
  }
  try {
    return thick_restarted_eigsh(op, options, initial_subspace);
  } catch (const QError& error) {
    if (error.code == ERR_NON_CONVERGENCE && dimension <= FULL_KRYLOV_DENSE_FALLBACK &&
        options.max_iterations >= dimension &&
        (options.krylov_dimension == 0 || options.krylov_dimension == dimension)) {
      Eigensystem result = dense_eigsh(op, options);
      result.iterations += error.iterations;
      return result;
    }
    throw;
  }
}

// eigsh / eigsh_with_initial / eigsh_with_initial_subspace (src/solve/mod.rs:2335-2417)
Eigensystem eigsh(const Operator& op, const EigshOptions& options,
                  const std::vector<std::vector<C64>>* initial_subspace) {
  if (op.rows != op.cols) fail(ERR_DIMENSION_MISMATCH, "eigsh requires a square operator");
  validate_options(options, op.rows);
  if (initial_subspace && !initial_subspace->empty()) {
    for (auto& v : *initial_subspace) {
      if (v.size() != op.rows) fail(ERR_DIMENSION_MISMATCH, "eigsh initial vector does not match the operator");
      for (auto& x : v)
        if (!std::isfinite(x.real()) || !std::isfinite(x.imag()))
          fail(ERR_INVALID_OPTIONS, "eigsh initial vector must contain only finite values");
      double n = vnorm(v);
      if (!std::isfinite(n) || n <= EPS) fail(ERR_INVALID_OPTIONS, "eigsh initial vector must have nonzero finite norm");
    }
  }
  if (use_dense_eigsh(op.rows, options)) return dense_eigsh(op, options);
  if (initial_subspace && initial_subspace->empty()) initial_subspace = nullptr;
  return expanding_lanczos_eigsh(op, options, initial_subspace);
}

// ----------------------------------------------------------------------------
// Exponential action: Al-Mohy--Higham Taylor plan (src/solve/mod.rs:14-248)
// ----------------------------------------------------------------------------
const std::pair<size_t, double> EXPM_TAYLOR_THETA[] = {
    {1, 2.29e-16}, {2, 2.58e-8}, {3, 1.39e-5}, {4, 3.40e-4}, {5, 2.40e-3}, {6, 9.07e-3},
    {7, 2.38e-2},  {8, 5.00e-2}, {9, 8.96e-2}, {10, 1.44e-1}, {11, 2.14e-1}, {12, 3.00e-1},
    {13, 4.00e-1}, {14, 5.14e-1}, {15, 6.41e-1}, {16, 7.81e-1}, {17, 9.31e-1}, {18, 1.09},
    {19, 1.26},    {20, 1.44},   {21, 1.62},   {22, 1.82},    {23, 2.01},    {24, 2.22},
    {25, 2.43},    {26, 2.64},   {27, 2.86},   {28, 3.08},    {29, 3.31},    {30, 3.54},
    {35, 4.7},     {40, 6.0},    {45, 7.2},    {50, 8.5},     {55, 9.9},
};

struct ExpmPlan {
  size_t dimension;
  C64 coefficient, shift;
  size_t degree, scaling;
  double tolerance;
};

// shifted_trace_and_one_norm (src/solve/mod.rs:59-104)
std::pair<C64, double> shifted_trace_and_one_norm(const Operator& op) {
  size_t n = op.rows;
  if (n == 0) return {C64(0.0, 0.0), 0.0};
  std::vector<C64> diagonal(n, C64(0.0, 0.0));
  std::vector<double> column_sums(n, 0.0);
  for (size_t r = 0; r < n; ++r)
    for (size_t p = op.row_ptr[r]; p < op.row_ptr[r + 1]; ++p) {
      size_t c = op.col_idx[p];
      if (r == c) diagonal[r] += op.values[p];
      else column_sums[c] += std::abs(op.values[p]);
    }
  C64 trace(0.0, 0.0);
  for (auto& d : diagonal) trace += d;
  C64 shift = trace / static_cast<double>(n);
  for (size_t c = 0; c < n; ++c) column_sums[c] += std::abs(diagonal[c] - shift);
  double maximum = 0.0;
  for (double s : column_sums) maximum = std::max(maximum, s);
  return {shift, maximum};
}

ExpmPlan expm_plan(const Operator& op, C64 coefficient, size_t max_degree, double tolerance, size_t max_substeps) {
  if (!std::isfinite(coefficient.real()) || !std::isfinite(coefficient.imag()) || max_degree == 0 ||
      !std::isfinite(tolerance) || tolerance <= 0.0 || max_substeps == 0)
    fail(ERR_INVALID_OPTIONS, "invalid exponential coefficient or numerical controls");
  auto [shift, one_norm] = shifted_trace_and_one_norm(op);
  double scaled = std::abs(coefficient) * one_norm;
  size_t degree = 0, scaling = 1;
  if (scaled != 0.0) {
    bool found = false;
    size_t best = 0;
    for (auto& [m, theta] : EXPM_TAYLOR_THETA) {
      if (m > max_degree) continue;
      size_t s = static_cast<size_t>(std::max(std::ceil(scaled / theta), 1.0));
      size_t cost = m * s;
      if (!found || cost < best) {
        found = true;
        best = cost;
        degree = m;
        scaling = s;
      }
    }
    if (!found) fail(ERR_INVALID_OPTIONS, "Taylor degree is below the minimum supported degree");
  }
  if (scaling > max_substeps) fail_nonconvergence(max_substeps, scaled);
  return {op.rows, coefficient, shift, degree, scaling, tolerance};
}

double inf_norm(const std::vector<C64>& v) {
  double m = 0.0;
  for (auto& x : v) m = std::max(m, std::abs(x));
  return m;
}

// ExpmActionPlan::apply (src/solve/mod.rs:198-247)
std::vector<C64> expm_apply(const ExpmPlan& plan, const Operator& op, const std::vector<C64>& initial) {
  if (initial.size() != plan.dimension) fail(ERR_DIMENSION_MISMATCH, "exponential plan, operator, and state dimensions do not match");
  if (std::abs(plan.coefficient) <= EPS || inf_norm(initial) == 0.0) return initial;
  C64 factor = plan.coefficient / static_cast<double>(plan.scaling);
  C64 eta = std::exp(factor * plan.shift);
  std::vector<C64> state = initial, applied(plan.dimension);
  for (size_t s = 0; s < plan.scaling; ++s) {
    std::vector<C64> term = state, sum = state;
    double previous = inf_norm(term);
    for (size_t order = 1; order <= plan.degree; ++order) {
      op.apply(term.data(), applied.data());
      C64 scale = factor / static_cast<double>(order);
      for (size_t i = 0; i < plan.dimension; ++i) applied[i] = scale * (applied[i] - plan.shift * term[i]);
      std::swap(term, applied);
      for (size_t i = 0; i < plan.dimension; ++i) sum[i] += term[i];
      double term_norm = inf_norm(term);
      if (previous + term_norm <= plan.tolerance * std::max(inf_norm(sum), std::numeric_limits<double>::min())) break;
      previous = term_norm;
    }
    for (size_t i = 0; i < plan.dimension; ++i) state[i] = eta * sum[i];
  }
  return state;
}

// ----------------------------------------------------------------------------
// Hermitian Krylov exponential action and adaptive evolution
// (src/solve/mod.rs:2909-3054 lanczos_projection(_real), 3056-3129 projected
// exponential coefficients/action, 3131-3195 residual amplitude and error
// bound, 3197-3316 evolve_hermitian_adaptive_grid, 3432-3454 expm_lanczos).
// ----------------------------------------------------------------------------
struct Projection {
  double initial_norm = 0.0;
  bool real = false;
  std::vector<std::vector<double>> rbasis;
  std::vector<std::vector<C64>> cbasis;
  double residual_beta = 0.0;
  std::vector<double> eigenvalues;
  std::vector<double> eigenvectors;  // column-major size x size
  size_t size() const { return real ? rbasis.size() : cbasis.size(); }
  double vec(size_t row, size_t col) const { return eigenvectors[row + size() * col]; }
};

double cnorm(const std::vector<C64>& v) {
  double s = 0.0;
  for (const C64& x : v) s += std::norm(x);
  return std::sqrt(s);
}

void finish_projection(Projection& p, const std::vector<double>& alphas, const std::vector<double>& betas) {
  const size_t size = p.size();
  std::vector<double> d(alphas.begin(), alphas.begin() + static_cast<long>(size));
  std::vector<double> e(size > 0 ? size - 1 : 0);
  for (size_t i = 0; i + 1 < size; ++i) e[i] = betas[i];
  tridiagonal_eigen(size, d, e, p.eigenvalues, p.eigenvectors);
}

// lanczos_projection_real (src/solve/mod.rs:2985-3054)
Projection lanczos_projection_real(const Operator& op, const std::vector<C64>& initial, size_t dimension) {
  Projection p;
  p.real = true;
  double sq = 0.0;
  for (const C64& x : initial) sq += x.real() * x.real();
  p.initial_norm = std::sqrt(sq);
  const size_t krylov = std::max<size_t>(std::min(dimension, initial.size()), 1);
  std::vector<double> first(initial.size());
  for (size_t i = 0; i < initial.size(); ++i) first[i] = initial[i].real() / p.initial_norm;
  p.rbasis.push_back(first);
  std::vector<double> alphas, betas, applied(initial.size());
  for (size_t it = 0; it < krylov; ++it) {
    op.apply_real(p.rbasis[it].data(), applied.data());
    double alpha = 0.0;
    for (size_t i = 0; i < applied.size(); ++i) alpha += p.rbasis[it][i] * applied[i];
    alphas.push_back(alpha);
    for (size_t i = 0; i < applied.size(); ++i) applied[i] -= alpha * p.rbasis[it][i];
    if (it > 0)
      for (size_t i = 0; i < applied.size(); ++i) applied[i] -= betas[it - 1] * p.rbasis[it - 1][i];
    double bsq = 0.0;
    for (double x : applied) bsq += x * x;
    const double beta = std::sqrt(bsq);
    p.residual_beta = beta;
    if (it + 1 == krylov || beta <= 1.0e-14) break;
    betas.push_back(beta);
    for (double& x : applied) x /= beta;
    p.rbasis.push_back(applied);
  }
  finish_projection(p, alphas, betas);
  return p;
}

// lanczos_projection (src/solve/mod.rs:2909-2983)
Projection lanczos_projection(const Operator& op, const std::vector<C64>& initial, size_t dimension) {
  Projection p;
  p.initial_norm = cnorm(initial);
  if (p.initial_norm <= EPS) return p;
  bool real_state = true;
  for (const C64& x : initial) real_state = real_state && x.imag() == 0.0;
  if (op.real && real_state) return lanczos_projection_real(op, initial, dimension);
  const size_t krylov = std::max<size_t>(std::min(dimension, initial.size()), 1);
  std::vector<C64> first = initial;
  for (C64& x : first) x /= p.initial_norm;
  p.cbasis.push_back(first);
  std::vector<double> alphas, betas;
  std::vector<C64> applied(initial.size());
  for (size_t it = 0; it < krylov; ++it) {
    op.apply(p.cbasis[it].data(), applied.data());
    C64 alpha(0.0, 0.0);
    for (size_t i = 0; i < applied.size(); ++i) alpha += std::conj(p.cbasis[it][i]) * applied[i];
    if (std::fabs(alpha.imag()) > 1.0e-10) fail(ERR_NON_HERMITIAN, "");
    alphas.push_back(alpha.real());
    for (size_t i = 0; i < applied.size(); ++i) applied[i] -= alpha.real() * p.cbasis[it][i];
    if (it > 0)
      for (size_t i = 0; i < applied.size(); ++i) applied[i] -= betas[it - 1] * p.cbasis[it - 1][i];
    const double beta = cnorm(applied);
    p.residual_beta = beta;
    if (it + 1 == krylov || beta <= 1.0e-14) break;
    betas.push_back(beta);
    for (C64& x : applied) x /= beta;
    p.cbasis.push_back(applied);
  }
  finish_projection(p, alphas, betas);
  return p;
}

// projected_exponential_coefficients (src/solve/mod.rs:3056-3075), Hamiltonian form
std::vector<C64> projected_coefficients(const Projection& p, double interval) {
  const size_t size = p.size();
  std::vector<C64> c(size, C64(0.0, 0.0));
  for (size_t e = 0; e < size; ++e) {
    const C64 weight = p.initial_norm * p.vec(0, e) * std::exp(C64(0.0, -interval * p.eigenvalues[e]));
    for (size_t b = 0; b < size; ++b) c[b] += p.vec(b, e) * weight;
  }
  return c;
}

// projected_exponential_action(_from_coefficients) (src/solve/mod.rs:3077-3129)
std::vector<C64> projected_action(const Projection& p, double interval, size_t n) {
  std::vector<C64> out(n, C64(0.0, 0.0));
  if (p.size() == 0) return out;
  const std::vector<C64> c = projected_coefficients(p, interval);
  for (size_t b = 0; b < p.size(); ++b) {
    if (p.real) {
      for (size_t i = 0; i < n; ++i) out[i] += C64(c[b].real() * p.rbasis[b][i], c[b].imag() * p.rbasis[b][i]);
    } else {
      for (size_t i = 0; i < n; ++i) out[i] += c[b] * p.cbasis[b][i];
    }
  }
  const double norm = cnorm(out);
  if (norm > EPS && std::isfinite(norm)) {
    const double scale = p.initial_norm / norm;
    for (C64& x : out) x *= scale;
  }
  return out;
}

// projected_residual_amplitude (src/solve/mod.rs:3131-3144)
double residual_amplitude(const Projection& p, double interval) {
  if (p.size() == 0) return 0.0;
  const size_t last = p.size() - 1;
  C64 a(0.0, 0.0);
  for (size_t e = 0; e < p.eigenvalues.size(); ++e)
    a += p.initial_norm * p.vec(0, e) * p.vec(last, e) * std::exp(C64(0.0, -interval * p.eigenvalues[e]));
  return std::abs(a);
}

// projected_exponential_error_bound (src/solve/mod.rs:3146-3195)
double error_bound(const Projection& p, double interval, size_t n) {
  const double duration = std::fabs(interval);
  if (duration <= EPS || p.size() == 0 || p.size() == n || p.residual_beta <= 1.0e-14) return 0.0;
  double lo = INFINITY, hi = -INFINITY;
  for (double v : p.eigenvalues) {
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  const double span = duration * std::max(hi - lo, 0.0);
  const size_t oscillations = static_cast<size_t>(std::min(std::ceil(span / M_PI), 60.0));
  size_t intervals = std::min<size_t>(16 + 4 * oscillations, 256);
  if (intervals % 2 != 0) ++intervals;
  const double direction = interval > 0 ? 1.0 : (interval < 0 ? -1.0 : 0.0);
  const double step = duration / static_cast<double>(intervals);
  double integral = 0.0;
  for (size_t i = 0; i <= intervals; ++i) {
    const double w = (i == 0 || i == intervals) ? 1.0 : (i % 2 == 0 ? 2.0 : 4.0);
    integral += w * residual_amplitude(p, direction * step * static_cast<double>(i));
  }
  return 1.25 * p.residual_beta * step * integral / 3.0;
}

struct EvolveDiagnostics {
  double lanczos_projections = 0, matrix_vector_products = 0, real_lanczos_projections = 0,
         real_matrix_vector_products = 0, accepted_substeps = 0, rejected_trial_intervals = 0,
         maximum_estimated_error = 0;
};

// EvolutionOptions::validate (src/solve/mod.rs:2510-2530)
void validate_evolution(const std::vector<double>& times, size_t krylov, double tolerance, size_t max_substeps) {
  bool ok = !times.empty();
  for (size_t i = 0; i < times.size(); ++i) {
    ok = ok && std::isfinite(times[i]);
    if (i > 0) ok = ok && !(times[i - 1] > times[i]);
  }
  if (!ok) fail(ERR_INVALID_OPTIONS, "times must be a nonempty finite nondecreasing grid");
  if (krylov == 0 || !std::isfinite(tolerance) || tolerance <= 0.0 || max_substeps == 0)
    fail(ERR_INVALID_OPTIONS, "evolution controls must be positive");
}

// evolve_hermitian_adaptive_grid (src/solve/mod.rs:3197-3316)
std::vector<std::vector<C64>> evolve_adaptive(const Operator& op, const std::vector<C64>& initial,
                                              const std::vector<double>& times, size_t krylov, double tolerance,
                                              size_t max_substeps, EvolveDiagnostics& d) {
  std::vector<std::vector<C64>> states;
  std::vector<C64> current = initial;
  double current_time = 0.0;
  size_t output = 0, substeps = 0;
  const double local_tolerance = tolerance / static_cast<double>(std::max<size_t>(times.size(), 1));
  const size_t n = initial.size();
  while (output < times.size()) {
    const double target = times[output];
    if (std::fabs(target - current_time) <= 16.0 * EPS * std::max(std::fabs(target), 1.0)) {
      states.push_back(current);
      current_time = target;
      ++output;
      continue;
    }
    if (substeps >= max_substeps) fail_nonconvergence(substeps, std::fabs(target - current_time));
    const Projection p = lanczos_projection(op, current, krylov);
    d.lanczos_projections += 1;
    d.matrix_vector_products += static_cast<double>(p.size());
    if (p.real) {
      d.real_lanczos_projections += 1;
      d.real_matrix_vector_products += static_cast<double>(p.size());
    }
    const double threshold = local_tolerance * std::max(cnorm(current), 1.0);
    std::vector<std::pair<double, std::vector<C64>>> accepted;
    for (size_t t = output; t < times.size(); ++t) {
      const double interval = times[t] - current_time;
      const double error = error_bound(p, interval, n);
      d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
      if (error > threshold) {
        d.rejected_trial_intervals += 1;
        break;
      }
      accepted.push_back({times[t], projected_action(p, interval, n)});
    }
    if (!accepted.empty()) {
      for (auto& a : accepted) states.push_back(a.second);
      current_time = accepted.back().first;
      current = accepted.back().second;
      output += accepted.size();
      ++substeps;
      d.accepted_substeps += 1;
      continue;
    }
    const double target_interval = target - current_time;
    const double direction = target_interval > 0 ? 1.0 : (target_interval < 0 ? -1.0 : 0.0);
    const double minimum = 16.0 * EPS * std::max(std::fabs(target), 1.0);
    double rejected = std::fabs(target_interval), accepted_mag = rejected;
    for (;;) {
      const double error = error_bound(p, direction * accepted_mag, n);
      d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
      if (error <= threshold || accepted_mag <= minimum) break;
      d.rejected_trial_intervals += 1;
      rejected = accepted_mag;
      accepted_mag *= 0.5;
    }
    if (accepted_mag > minimum && rejected > accepted_mag) {
      for (int i = 0; i < 8; ++i) {
        const double trial = 0.5 * (accepted_mag + rejected);
        const double error = error_bound(p, direction * trial, n);
        d.maximum_estimated_error = std::max(d.maximum_estimated_error, error);
        if (error <= threshold) {
          accepted_mag = trial;
        } else {
          d.rejected_trial_intervals += 1;
          rejected = trial;
        }
      }
    }
    const double interval = direction * accepted_mag;
    current_time += interval;
    current = projected_action(p, interval, n);
    ++substeps;
    d.accepted_substeps += 1;
  }
  return states;
}

// ----------------------------------------------------------------------------
// Cross-sector action and spectral functions (src/operator/mod.rs:2305-2351
// apply_sector_shift; src/dynamics/mod.rs:903-1021 SpectrumOptions and
// spectral_function; src/solve/mod.rs:2886-2907 lanczos_spectral_measure,
// 558-583 hermitian_eigenpairs_all).
// ----------------------------------------------------------------------------
std::vector<C64> apply_sector_shift(const SpinBasis& source, const SpinBasis& target, const std::vector<Term>& terms,
                                    const std::vector<C64>& input) {
  if (input.size() != source.len())
    fail(ERR_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
  std::vector<C64> output(target.len(), C64(0.0, 0.0));
  for (size_t column = 0; column < input.size(); ++column) {
    const C64 value = input[column];
    if (std::abs(value) <= EPS) continue;
    const u128 state = source.states[column];
    const size_t orbit = source.transition_orbit_size(state);
    for (const Term& term : terms)
      for (const Coupling& coupling : term.couplings)
        source.visit_transitions(state, term.symbols, coupling.sites, [&](u128 unreduced, C64 local) {
          size_t row;
          C64 reduction;
          if (!target.index_transition(unreduced, orbit, &row, &reduction)) return;
          output[row] += value * coupling.coefficient * local * reduction;
        });
  }
  return output;
}

// SpectrumOptions::validate (src/dynamics/mod.rs:945-962)
void validate_spectrum(const std::vector<double>& frequencies, double reference_energy, double broadening,
                       size_t krylov, double tolerance) {
  bool ok = !frequencies.empty() && std::isfinite(reference_energy) && std::isfinite(broadening) &&
            broadening > 0.0 && krylov > 0 && std::isfinite(tolerance) && tolerance > 0.0;
  for (double f : frequencies) ok = ok && std::isfinite(f);
  if (!ok) fail(ERR_INVALID_OPTIONS, "invalid spectrum frequency grid or numerical controls");
}

// spectral_function on the probed vector `created` (= probe |source>):
// all eigenpairs when the target has at most 128 states, else the Lanczos
// spectral measure of `krylov` steps; Lorentzians of width `broadening`.
std::vector<double> spectral_function(const Operator& target, const std::vector<C64>& created,
                                      const std::vector<double>& frequencies, double reference_energy,
                                      double broadening, size_t krylov, double tolerance) {
  validate_spectrum(frequencies, reference_energy, broadening, krylov, tolerance);
  if (target.rows != target.cols || created.size() != target.rows)
    fail(ERR_DIMENSION_MISMATCH, "target Hamiltonian, source, and probe shapes are incompatible");
  std::vector<double> energies, weights;
  const size_t n = target.rows;
  if (n <= 128) {
    std::vector<C64> dense(n * n, C64(0.0, 0.0));
    for (size_t r = 0; r < n; ++r)
      for (size_t p = target.row_ptr[r]; p < target.row_ptr[r + 1]; ++p) dense[r * n + target.col_idx[p]] += target.values[p];
    for (size_t r = 0; r < n; ++r)
      for (size_t c = 0; c < n; ++c)
        if (std::abs(dense[r * n + c] - std::conj(dense[c * n + r])) > 1.0e-12) fail(ERR_NON_HERMITIAN, "");
    std::vector<C64> vectors;
    hermitian_jacobi(n, dense, energies, vectors);
    for (size_t e = 0; e < n; ++e) {
      C64 overlap(0.0, 0.0);
      for (size_t i = 0; i < n; ++i) overlap += std::conj(vectors[i + n * e]) * created[i];
      weights.push_back(std::norm(overlap));
    }
  } else {
    const Projection p = lanczos_projection(target, created, krylov);
    energies = p.eigenvalues;
    for (size_t e = 0; e < p.eigenvalues.size(); ++e)
      weights.push_back(p.initial_norm * p.initial_norm * p.vec(0, e) * p.vec(0, e));
  }
  std::vector<double> out;
  const double pi = 3.14159265358979323846;
  for (double frequency : frequencies) {
    double sum = 0.0;
    for (size_t e = 0; e < energies.size(); ++e) {
      const double detuning = frequency + reference_energy - energies[e];
      sum += weights[e] * broadening / (pi * (detuning * detuning + broadening * broadening));
    }
    out.push_back(sum);
  }
  return out;
}

// ----------------------------------------------------------------------------
// Full Lanczos decomposition and thermal Lanczos (src/solve/mod.rs:2674-2857
// lanczos_iter / lanczos_full / lanczos_ritz, 3457-3568 thermal static
// iteration, 3575-3940 projected observables and FTLM/LTLM contractions).
// Complex arithmetic throughout, like the reference.
// ----------------------------------------------------------------------------
struct LanczosFull {
  double initial_norm = 0.0;
  std::vector<std::vector<C64>> basis;
  std::vector<double> diagonal, off_diagonal;
};

// LanczosOptions::validate (src/solve/mod.rs:2590-2597)
void validate_lanczos(size_t krylov, double tolerance) {
  if (krylov == 0 || !std::isfinite(tolerance) || tolerance <= 0.0)
    fail(ERR_INVALID_OPTIONS, "Lanczos dimension and tolerance must be positive");
}

C64 cinner(const std::vector<C64>& a, const std::vector<C64>& b) {
  C64 s(0.0, 0.0);
  for (size_t i = 0; i < a.size(); ++i) s += std::conj(a[i]) * b[i];
  return s;
}

// lanczos_full over LanczosIter::next (src/solve/mod.rs:2694-2813): three-term
// step, then modified Gram-Schmidt against every earlier vector and the
// current one, repeated once when the norm fell to 1/sqrt(2) of its value
// before (DGKS); stops after `krylov` vectors or when beta <= tolerance.
LanczosFull lanczos_full(const Operator& op, const std::vector<C64>& initial, size_t krylov, double tolerance) {
  validate_lanczos(krylov, tolerance);
  if (op.rows != op.cols || initial.size() != op.rows)
    fail(ERR_DIMENSION_MISMATCH, "Lanczos operator and initial vector do not match");
  LanczosFull f;
  f.initial_norm = cnorm(initial);
  if (!std::isfinite(f.initial_norm) || f.initial_norm <= EPS) fail(ERR_NON_CONVERGENCE, "initial vector is zero");
  std::vector<C64> current = initial, previous, applied(initial.size());
  for (C64& x : current) x /= f.initial_norm;
  double previous_beta = 0.0;
  std::vector<double> betas;
  for (size_t index = 0; index < krylov; ++index) {
    op.apply(current.data(), applied.data());
    const C64 alpha = cinner(current, applied);
    if (std::fabs(alpha.imag()) > std::max(tolerance, 1.0e-10)) fail(ERR_NON_HERMITIAN, "");
    for (size_t i = 0; i < applied.size(); ++i) applied[i] -= alpha.real() * current[i];
    if (!previous.empty())
      for (size_t i = 0; i < applied.size(); ++i) applied[i] -= previous_beta * previous[i];
    auto sweep = [&] {
      for (size_t b = 0; b <= f.basis.size(); ++b) {
        const std::vector<C64>& q = b < f.basis.size() ? f.basis[b] : current;
        const C64 c = cinner(q, applied);
        for (size_t i = 0; i < applied.size(); ++i) applied[i] -= c * q[i];
      }
    };
    const double before = cnorm(applied);
    sweep();
    if (before > EPS && cnorm(applied) <= DGKS_THRESHOLD * before) sweep();
    const double beta = cnorm(applied);
    f.diagonal.push_back(alpha.real());
    betas.push_back(beta);
    f.basis.push_back(current);
    if (index + 1 < krylov && beta > tolerance) {
      for (C64& x : applied) x /= beta;
      previous = current;
      current = applied;
      previous_beta = beta;
    } else {
      break;
    }
  }
  f.off_diagonal.assign(betas.begin(), betas.end() - 1);
  return f;
}

// lanczos_ritz (src/solve/mod.rs:2818-2857): ascending Ritz values and the
// eigenvectors of the tridiagonal, vectors[column][row].
struct LanczosRitz {
  LanczosFull d;
  std::vector<double> values;
  std::vector<std::vector<double>> vectors;
};

LanczosRitz lanczos_ritz(const Operator& op, const std::vector<C64>& initial, size_t krylov, double tolerance) {
  LanczosRitz r;
  r.d = lanczos_full(op, initial, krylov, tolerance);
  const size_t m = r.d.diagonal.size();
  std::vector<double> w, z;
  tridiagonal_eigen(m, r.d.diagonal, r.d.off_diagonal, w, z);
  std::vector<size_t> order(m);
  for (size_t i = 0; i < m; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return w[a] < w[b]; });
  for (size_t c : order) {
    r.values.push_back(w[c]);
    r.vectors.emplace_back(z.begin() + static_cast<long>(m * c), z.begin() + static_cast<long>(m * (c + 1)));
  }
  return r;
}

void validate_inverse_temperatures(const std::vector<double>& betas, bool nonnegative) {
  bool ok = !betas.empty();
  for (double b : betas) ok = ok && std::isfinite(b) && (!nonnegative || b >= 0.0);
  if (!ok) fail(ERR_INVALID_OPTIONS, "inverse temperatures must be nonempty, finite, and nonnegative");
}

// thermal_lanczos_iteration (src/solve/mod.rs:3464-3540), shared by
// ftlm_static_iteration and ltlm_static_iteration (3543-3568):
// weights |v|^2 V[0,i]^2, log Z = ln(D / |v|^2) - beta E_min + ln sum w e^{-beta (E - E_min)}.
void thermal_iteration(const Operator& op, const std::vector<C64>& initial, const std::vector<double>& betas,
                       size_t krylov, double tolerance, std::vector<double>& log_partition,
                       std::vector<double>& mean_energy, size_t& size) {
  validate_lanczos(krylov, tolerance);
  validate_inverse_temperatures(betas, true);
  const LanczosRitz r = lanczos_ritz(op, initial, krylov, tolerance);
  size = r.values.size();
  const double norm_sq = r.d.initial_norm * r.d.initial_norm;
  std::vector<double> weights(size);
  double e_min = INFINITY;
  for (size_t i = 0; i < size; ++i) {
    weights[i] = norm_sq * r.vectors[i][0] * r.vectors[i][0];
    e_min = std::min(e_min, r.values[i]);
  }
  log_partition.clear();
  mean_energy.clear();
  for (double beta : betas) {
    double z = 0.0, e = 0.0;
    for (size_t i = 0; i < size; ++i) {
      const double b = weights[i] * std::exp(-beta * (r.values[i] - e_min));
      z += b;
      e += b * r.values[i];
    }
    if (z <= EPS) fail(ERR_NON_CONVERGENCE, "projected partition function vanished");
    log_partition.push_back(std::log(static_cast<double>(op.rows) / norm_sq) - beta * e_min + std::log(z));
    mean_energy.push_back(e / z);
  }
}

// project_thermal_observables (src/solve/mod.rs:3813-3856): FTLM keeps
// <q_i|A|q_0>; LTLM keeps <q_j|A|q_i> at i * m + j.
std::vector<C64> project_observable(const LanczosRitz& r, const Operator& a, bool ltlm) {
  const size_t m = r.d.basis.size();
  if (m == 0 || a.rows != r.d.basis[0].size() || a.cols != a.rows)
    fail(ERR_DIMENSION_MISMATCH, "thermal observables require unique names and matching square shapes");
  std::vector<C64> out, applied(a.rows);
  for (size_t input = 0; input < (ltlm ? m : 1); ++input) {
    a.apply(r.d.basis[input].data(), applied.data());
    for (size_t bra = 0; bra < m; ++bra) out.push_back(cinner(r.d.basis[bra], applied));
  }
  return out;
}

// ftlm_projected_contraction (src/solve/mod.rs:3646-3694): values[o][b] and identity[b].
void ftlm_contraction(const LanczosRitz& r, const std::vector<std::vector<C64>>& projected,
                      const std::vector<double>& betas, std::vector<std::vector<C64>>& values,
                      std::vector<double>& identity) {
  const size_t m = r.values.size();
  values.assign(projected.size(), {});
  identity.clear();
  for (double beta : betas) {
    std::vector<double> coefficient(m, 0.0);
    for (size_t row = 0; row < m; ++row)
      for (size_t e = 0; e < m; ++e)
        coefficient[row] += r.vectors[e][row] * r.vectors[e][0] * std::exp(-beta * r.values[e]);
    identity.push_back(coefficient[0]);
    for (size_t o = 0; o < projected.size(); ++o) {
      C64 s(0.0, 0.0);
      for (size_t row = 0; row < m; ++row) s += projected[o][row] * coefficient[row];
      values[o].push_back(s);
    }
  }
}

// ltlm_effective_dimension and ltlm_projected_contraction (src/solve/mod.rs:3696-3778)
void ltlm_contraction(const LanczosRitz& r, const std::vector<std::vector<C64>>& projected,
                      const std::vector<double>& betas, std::vector<std::vector<C64>>& values,
                      std::vector<double>& identity) {
  const size_t full = r.values.size();
  double beta_min = INFINITY, first_max = 0.0;
  for (double b : betas) beta_min = std::min(beta_min, b);
  for (const auto& v : r.vectors) first_max = std::max(first_max, std::fabs(v[0]));
  size_t m = full;
  for (size_t e = 0; e < full; ++e)
    if (std::exp(-r.values[e] * beta_min) * first_max < EPS) {
      m = e;
      break;
    }
  if (m == 0) fail(ERR_NON_CONVERGENCE, "no Ritz state carries Boltzmann weight");
  identity.clear();
  for (double beta : betas) {
    double s = 0.0;
    for (size_t e = 0; e < m; ++e) s += r.vectors[e][0] * r.vectors[e][0] * std::exp(-beta * r.values[e]);
    identity.push_back(s);
  }
  values.assign(projected.size(), {});
  for (size_t o = 0; o < projected.size(); ++o) {
    std::vector<C64> t(m * m, C64(0.0, 0.0));
    for (size_t left = 0; left < m; ++left)
      for (size_t right = 0; right < m; ++right) {
        C64 s(0.0, 0.0);
        for (size_t in = 0; in < m; ++in)
          for (size_t bra = 0; bra < m; ++bra)
            s += r.vectors[left][in] * projected[o][in * full + bra] * r.vectors[right][bra];
        t[left * m + right] = s;
      }
    for (double beta : betas) {
      std::vector<double> w(m);
      for (size_t e = 0; e < m; ++e) w[e] = r.vectors[e][0] * std::exp(-0.5 * beta * r.values[e]);
      C64 s(0.0, 0.0);
      for (size_t left = 0; left < m; ++left)
        for (size_t right = 0; right < m; ++right) s += w[left] * t[left * m + right] * w[right];
      values[o].push_back(s);
    }
  }
}

// ----------------------------------------------------------------------------
// C ABI used by the tests (ctypes).
// ----------------------------------------------------------------------------
thread_local std::string g_last_error;

template <typename F>
int guarded(F&& body) {
  try {
    body();
    g_last_error.clear();
    return 0;
  } catch (const QError& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal state error: ") + e.what();
    return ERR_INTERNAL_STATE;
  }
}

std::vector<Term> decode_terms(int n_terms, const int* arity, const char* symbols, const int* n_couplings,
                               const double* coefficients, const int* sites) {
  std::vector<Term> terms(static_cast<size_t>(n_terms));
  size_t symbol_cursor = 0, coupling_cursor = 0, site_cursor = 0;
  for (int t = 0; t < n_terms; ++t) {
    Term& term = terms[static_cast<size_t>(t)];
    for (int a = 0; a < arity[t]; ++a) term.symbols.push_back(symbols[symbol_cursor++]);
    term.label = std::string(term.symbols.begin(), term.symbols.end());
    for (int c = 0; c < n_couplings[t]; ++c) {
      Coupling coupling;
      coupling.coefficient = C64(coefficients[2 * coupling_cursor], coefficients[2 * coupling_cursor + 1]);
      ++coupling_cursor;
      for (int a = 0; a < arity[t]; ++a) coupling.sites.push_back(static_cast<size_t>(sites[site_cursor++]));
      term.couplings.push_back(std::move(coupling));
    }
  }
  return terms;
}

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_last_error.c_str(); }

int oracle_basis_create(int sites, int up, int has_momentum, int momentum, int parity, int normalization,
                        void** out) {
  return guarded([&] {
    if (sites <= 0 || sites > 128) fail(ERR_UNSUPPORTED_BACKEND, "the oracle supports 1..128 sites");
    *out = build_spin_basis(static_cast<size_t>(sites), up, has_momentum != 0, momentum, parity, normalization).release();
  });
}

void oracle_basis_free(void* basis) { delete static_cast<SpinBasis*>(basis); }

long long oracle_basis_dim(void* basis) { return static_cast<long long>(static_cast<SpinBasis*>(basis)->len()); }

int oracle_basis_states(void* handle, uint64_t* lo, uint64_t* hi, uint64_t* orbit) {
  return guarded([&] {
    auto* basis = static_cast<SpinBasis*>(handle);
    for (size_t i = 0; i < basis->len(); ++i) {
      if (lo) lo[i] = static_cast<uint64_t>(basis->states[i]);
      if (hi) hi[i] = static_cast<uint64_t>(basis->states[i] >> 64);
      if (orbit) orbit[i] = basis->orbit_lengths[i];
    }
  });
}

// Reduction image of one physical state: returns 1 if the state belongs to a
// compatible orbit, 0 otherwise.
int oracle_basis_image(void* handle, uint64_t lo, uint64_t hi, uint64_t* rep_lo, uint64_t* rep_hi,
                       double* phase, uint64_t* orbit) {
  auto* basis = static_cast<SpinBasis*>(handle);
  u128 state = (static_cast<u128>(hi) << 64) | lo;
  if (!basis->symmetric()) {
    size_t idx;
    if (!basis->index(state, &idx)) return 0;
    *rep_lo = lo; *rep_hi = hi; phase[0] = 1.0; phase[1] = 0.0; *orbit = 1;
    return 1;
  }
  auto it = basis->lookup.find(state);
  if (it == basis->lookup.end()) return 0;
  *rep_lo = static_cast<uint64_t>(it->second.representative);
  *rep_hi = static_cast<uint64_t>(it->second.representative >> 64);
  phase[0] = it->second.phase.real();
  phase[1] = it->second.phase.imag();
  *orbit = it->second.orbit_size;
  return 1;
}

// Reduction images of physical states by the reference's per-orbit rule
// alone: the orbit of each state, its minimum, and the projection of that
// orbit (project_orbit), without building the sector. For sectors too large
// for the full lookup. Outputs per state: representative (lo/hi words),
// phase (2 doubles) and orbit size (0 when the orbit is not in the sector).
int oracle_orbit_images(int sites, int has_momentum, int momentum, int parity, long long n, const uint64_t* lo,
                        const uint64_t* hi, uint64_t* rep_lo, uint64_t* rep_hi, double* phase, uint64_t* orbit) {
  return guarded([&] {
    const size_t L = static_cast<size_t>(sites);
    const long normalized = has_momentum ? ((momentum % sites) + sites) % sites : 0;
    const size_t translations = has_momentum ? L : 1;
    for (long long i = 0; i < n; ++i) {
      const u128 state = (static_cast<u128>(hi ? hi[i] : 0) << 64) | lo[i];
      u128 representative = state;
      for (size_t shift = 0; shift < translations; ++shift) {
        u128 translated = rotate_lattice_state(state, shift, L);
        representative = std::min(representative, translated);
        if (parity != 0) representative = std::min(representative, reflect_lattice_state(translated, L));
      }
      std::unordered_map<u128, SymmetryImage, U128Hash> images;
      size_t orbit_size = 0;
      const bool kept = project_orbit(representative, L, translations, normalized, parity, has_momentum != 0,
                                      images, &orbit_size);
      auto it = images.find(state);
      if (!kept || it == images.end()) {
        rep_lo[i] = rep_hi[i] = 0;
        phase[2 * i] = phase[2 * i + 1] = 0.0;
        orbit[i] = 0;
        continue;
      }
      rep_lo[i] = static_cast<uint64_t>(it->second.representative);
      rep_hi[i] = static_cast<uint64_t>(it->second.representative >> 64);
      phase[2 * i] = it->second.phase.real();
      phase[2 * i + 1] = it->second.phase.imag();
      orbit[i] = it->second.orbit_size;
    }
  });
}

int oracle_operator_build(void* basis, int n_terms, const int* arity, const char* symbols, const int* n_couplings,
                          const double* coefficients, const int* sites, int check_hermitian, int check_particles,
                          void** out) {
  return guarded([&] {
    auto terms = decode_terms(n_terms, arity, symbols, n_couplings, coefficients, sites);
    *out = build_operator(*static_cast<SpinBasis*>(basis), terms, check_hermitian != 0, check_particles != 0).release();
  });
}

int oracle_operator_from_triplets(long long n, long long nnz, const int64_t* rows, const int64_t* cols,
                                  const double* values, void** out) {
  return guarded([&] {
    std::vector<size_t> r(static_cast<size_t>(nnz)), c(static_cast<size_t>(nnz));
    std::vector<C64> v(static_cast<size_t>(nnz));
    for (long long i = 0; i < nnz; ++i) {
      r[static_cast<size_t>(i)] = static_cast<size_t>(rows[i]);
      c[static_cast<size_t>(i)] = static_cast<size_t>(cols[i]);
      v[static_cast<size_t>(i)] = C64(values[2 * i], values[2 * i + 1]);
    }
    *out = operator_from_triplets(static_cast<size_t>(n), r, c, v).release();
  });
}

void oracle_operator_free(void* op) { delete static_cast<Operator*>(op); }

long long oracle_operator_dim(void* op) { return static_cast<long long>(static_cast<Operator*>(op)->rows); }
long long oracle_operator_nnz(void* op) { return static_cast<long long>(static_cast<Operator*>(op)->values.size()); }
int oracle_operator_is_real(void* op) { return static_cast<Operator*>(op)->real ? 1 : 0; }

int oracle_operator_csr(void* handle, int64_t* row_ptr, int64_t* cols, double* values) {
  return guarded([&] {
    auto* op = static_cast<Operator*>(handle);
    for (size_t i = 0; i <= op->rows; ++i) row_ptr[i] = static_cast<int64_t>(op->row_ptr[i]);
    for (size_t i = 0; i < op->values.size(); ++i) {
      cols[i] = static_cast<int64_t>(op->col_idx[i]);
      values[2 * i] = op->values[i].real();
      values[2 * i + 1] = op->values[i].imag();
    }
  });
}

// y = H x for complex-interleaved vectors.
int oracle_operator_apply(void* handle, const double* x, double* y) {
  return guarded([&] {
    auto* op = static_cast<Operator*>(handle);
    op->apply(reinterpret_cast<const C64*>(x), reinterpret_cast<C64*>(y));
  });
}

int oracle_deterministic_start(long long n, uint64_t seed, double* out) {
  return guarded([&] {
    auto v = deterministic_start(static_cast<size_t>(n), seed);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i].real();
  });
}

// eigsh with optional initial subspace (n_initial vectors of length dim,
// complex interleaved). Output arrays hold `eigenpairs` entries; eigenvectors
// (nullable) hold eigenpairs*dim complex values. counters[0..2] receive
// iterations, reorthogonalization passes, conditional second passes.
int oracle_eigsh(void* handle, long long eigenpairs, int target, double shift, long long krylov_dimension,
                 double tolerance, long long max_iterations, uint64_t seed, const double* initial, int n_initial,
                 double* eigenvalues, double* residuals, double* eigenvectors, long long* counters) {
  return guarded([&] {
    auto* op = static_cast<Operator*>(handle);
    EigshOptions o;
    o.eigenpairs = static_cast<size_t>(eigenpairs);
    o.target = target;
    o.shift = shift;
    o.krylov_dimension = static_cast<size_t>(krylov_dimension);
    o.tolerance = tolerance;
    o.max_iterations = static_cast<size_t>(max_iterations);
    o.seed = seed;
    std::vector<std::vector<C64>> subspace;
    for (int k = 0; k < n_initial; ++k) {
      const C64* base = reinterpret_cast<const C64*>(initial) + static_cast<size_t>(k) * op->rows;
      subspace.emplace_back(base, base + op->rows);
    }
    Eigensystem result = eigsh(*op, o, n_initial > 0 ? &subspace : nullptr);
    for (size_t i = 0; i < result.eigenvalues.size(); ++i) {
      eigenvalues[i] = result.eigenvalues[i];
      residuals[i] = result.residuals[i];
      if (eigenvectors)
        for (size_t j = 0; j < op->rows; ++j) {
          eigenvectors[2 * (i * op->rows + j)] = result.eigenvectors[i][j].real();
          eigenvectors[2 * (i * op->rows + j) + 1] = result.eigenvectors[i][j].imag();
        }
    }
    counters[0] = static_cast<long long>(result.iterations);
    counters[1] = static_cast<long long>(result.reorthogonalization_passes);
    counters[2] = static_cast<long long>(result.conditional_second_passes);
  });
}

int oracle_expm_plan(void* handle, double coef_re, double coef_im, long long max_degree, double tolerance,
                     long long max_substeps, long long* degree, long long* scaling, double* shift, double* one_norm) {
  return guarded([&] {
    auto* op = static_cast<Operator*>(handle);
    ExpmPlan plan = expm_plan(*op, C64(coef_re, coef_im), static_cast<size_t>(max_degree), tolerance,
                              static_cast<size_t>(max_substeps));
    *degree = static_cast<long long>(plan.degree);
    *scaling = static_cast<long long>(plan.scaling);
    shift[0] = plan.shift.real();
    shift[1] = plan.shift.imag();
    if (one_norm) *one_norm = shifted_trace_and_one_norm(*op).second;
  });
}

int oracle_expm_apply(void* handle, double coef_re, double coef_im, long long max_degree, double tolerance,
                      long long max_substeps, const double* input, double* output) {
  return guarded([&] {
    auto* op = static_cast<Operator*>(handle);
    ExpmPlan plan = expm_plan(*op, C64(coef_re, coef_im), static_cast<size_t>(max_degree), tolerance,
                              static_cast<size_t>(max_substeps));
    std::vector<C64> in(reinterpret_cast<const C64*>(input), reinterpret_cast<const C64*>(input) + op->rows);
    auto result = expm_apply(plan, *op, in);
    for (size_t i = 0; i < result.size(); ++i) {
      output[2 * i] = result[i].real();
      output[2 * i + 1] = result[i].imag();
    }
  });
}

// Dense Hermitian eigensolver exposed for direct checks against numpy.
int oracle_hermitian_eigen(long long n, const double* a, double* values, double* vectors) {
  return guarded([&] {
    std::vector<C64> m(reinterpret_cast<const C64*>(a), reinterpret_cast<const C64*>(a) + n * n);
    std::vector<double> w;
    std::vector<C64> v;
    hermitian_jacobi(static_cast<size_t>(n), m, w, v);
    for (long long i = 0; i < n; ++i) values[i] = w[static_cast<size_t>(i)];
    for (long long i = 0; i < n * n; ++i) {
      vectors[2 * i] = v[static_cast<size_t>(i)].real();
      vectors[2 * i + 1] = v[static_cast<size_t>(i)].imag();
    }
  });
}

// evolve (src/solve/mod.rs:3374-3406) with hamiltonian = true: `initial` and
// each of the n_times output states are interleaved complex vectors.
// diagnostics[7]: EvolutionDiagnostics fields in declaration order.
int oracle_evolve(void* handle, const double* initial, long long n_times, const double* times, long long krylov,
                  double tolerance, long long max_substeps, double* states, double* diagnostics) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(handle);
    std::vector<double> grid(times, times + n_times);
    validate_evolution(grid, static_cast<size_t>(std::max(krylov, 0LL)), tolerance,
                       static_cast<size_t>(std::max(max_substeps, 0LL)));
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(initial[2 * i], initial[2 * i + 1]);
    EvolveDiagnostics d;
    auto out = evolve_adaptive(op, v, grid, static_cast<size_t>(krylov), tolerance, static_cast<size_t>(max_substeps), d);
    for (size_t t = 0; t < out.size(); ++t)
      for (size_t i = 0; i < op.rows; ++i) {
        states[2 * (t * op.rows + i)] = out[t][i].real();
        states[2 * (t * op.rows + i) + 1] = out[t][i].imag();
      }
    const double fields[7] = {d.lanczos_projections, d.matrix_vector_products, d.real_lanczos_projections,
                              d.real_matrix_vector_products, d.accepted_substeps, d.rejected_trial_intervals,
                              d.maximum_estimated_error};
    for (int i = 0; i < 7; ++i) diagnostics[i] = fields[i];
  });
}

// expm_lanczos (src/solve/mod.rs:3432-3454): exp(-i t H) v from one projection.
int oracle_expm_lanczos(void* handle, const double* initial, double time, long long krylov, double* out) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(handle);
    if (krylov <= 0) fail(ERR_INVALID_OPTIONS, "Lanczos dimension and tolerance must be positive");
    if (!std::isfinite(time)) fail(ERR_INVALID_OPTIONS, "exponential time must be finite");
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(initial[2 * i], initial[2 * i + 1]);
    const Projection p = lanczos_projection(op, v, static_cast<size_t>(krylov));
    const std::vector<C64> r = projected_action(p, time, op.rows);
    for (size_t i = 0; i < op.rows; ++i) {
      out[2 * i] = r[i].real();
      out[2 * i + 1] = r[i].imag();
    }
  });
}

int oracle_tridiagonal_eigen(long long n, const double* diag, const double* off, double* values, double* vectors) {
  return guarded([&] {
    std::vector<double> d(diag, diag + n), e(off, off + (n > 0 ? n - 1 : 0)), w, z;
    tridiagonal_eigen(static_cast<size_t>(n), d, e, w, z);
    for (long long i = 0; i < n; ++i) values[i] = w[static_cast<size_t>(i)];
    for (long long i = 0; i < n * n; ++i) vectors[i] = z[static_cast<size_t>(i)];
  });
}

// lanczos_ritz (src/solve/mod.rs:2818-2857). Outputs sized for `krylov`
// vectors: basis[krylov][dim] interleaved complex, diagonal[krylov],
// off_diagonal[krylov - 1], values[krylov], vectors[krylov * krylov] with
// vectors[column * size + row]; *size receives the decomposition length.
int oracle_lanczos_ritz(void* handle, const double* initial, long long krylov, double tolerance, long long* size,
                        double* initial_norm, double* basis, double* diagonal, double* off_diagonal, double* values,
                        double* vectors) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(handle);
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(initial[2 * i], initial[2 * i + 1]);
    const LanczosRitz r = lanczos_ritz(op, v, static_cast<size_t>(std::max(krylov, 0LL)), tolerance);
    const size_t m = r.values.size();
    *size = static_cast<long long>(m);
    *initial_norm = r.d.initial_norm;
    for (size_t b = 0; b < m; ++b) {
      for (size_t i = 0; i < op.rows; ++i) {
        basis[2 * (b * op.rows + i)] = r.d.basis[b][i].real();
        basis[2 * (b * op.rows + i) + 1] = r.d.basis[b][i].imag();
      }
      diagonal[b] = r.d.diagonal[b];
      if (b + 1 < m) off_diagonal[b] = r.d.off_diagonal[b];
      values[b] = r.values[b];
      for (size_t row = 0; row < m; ++row) vectors[b * m + row] = r.vectors[b][row];
    }
  });
}

// ftlm_static_iteration / ltlm_static_iteration (src/solve/mod.rs:3543-3568)
int oracle_thermal_iteration(void* handle, const double* initial, long long n_betas, const double* betas,
                             long long krylov, double tolerance, double* log_partition, double* mean_energy,
                             long long* size) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(handle);
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(initial[2 * i], initial[2 * i + 1]);
    std::vector<double> lz, e;
    size_t m = 0;
    thermal_iteration(op, v, std::vector<double>(betas, betas + std::max(n_betas, 0LL)),
                      static_cast<size_t>(std::max(krylov, 0LL)), tolerance, lz, e, m);
    for (size_t b = 0; b < lz.size(); ++b) {
      log_partition[b] = lz[b];
      mean_energy[b] = e[b];
    }
    *size = static_cast<long long>(m);
  });
}

// ftlm_observable_iteration / ltlm_observable_iteration (src/solve/mod.rs:3858-3898):
// method 0 FTLM, 1 LTLM; values[o][b] interleaved complex, identity[b].
int oracle_thermal_observables(void* handle, const double* initial, long long krylov, double tolerance, int method,
                               long long n_observables, void* const* observables, long long n_betas,
                               const double* betas, double* values, double* identity) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(handle);
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(initial[2 * i], initial[2 * i + 1]);
    const LanczosRitz r = lanczos_ritz(op, v, static_cast<size_t>(std::max(krylov, 0LL)), tolerance);
    if (n_observables <= 0) fail(ERR_INVALID_OPTIONS, "thermal observables must be nonempty");
    std::vector<double> grid(betas, betas + std::max(n_betas, 0LL));
    validate_inverse_temperatures(grid, false);
    std::vector<std::vector<C64>> projected;
    for (long long o = 0; o < n_observables; ++o)
      projected.push_back(project_observable(r, *static_cast<const Operator*>(observables[o]), method == 1));
    std::vector<std::vector<C64>> out;
    std::vector<double> id;
    if (method == 1)
      ltlm_contraction(r, projected, grid, out, id);
    else
      ftlm_contraction(r, projected, grid, out, id);
    for (size_t o = 0; o < out.size(); ++o)
      for (size_t b = 0; b < grid.size(); ++b) {
        values[2 * (o * grid.size() + b)] = out[o][b].real();
        values[2 * (o * grid.size() + b) + 1] = out[o][b].imag();
      }
    for (size_t b = 0; b < grid.size(); ++b) identity[b] = id[b];
  });
}

// apply_sector_shift (src/operator/mod.rs:2305-2351): input on `source`,
// output on `target` (interleaved complex).
int oracle_sector_shift(void* source, void* target, int n_terms, const int* arity, const char* symbols,
                        const int* n_couplings, const double* coefficients, const int* sites, long long n_input,
                        const double* input, long long n_output, double* output) {
  return guarded([&] {
    const SpinBasis& s = *static_cast<SpinBasis*>(source);
    const SpinBasis& t = *static_cast<SpinBasis*>(target);
    auto terms = decode_terms(n_terms, arity, symbols, n_couplings, coefficients, sites);
    if (n_output != static_cast<long long>(t.len()))
      fail(ERR_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
    std::vector<C64> x(static_cast<size_t>(std::max(n_input, 0LL)));
    for (size_t i = 0; i < x.size(); ++i) x[i] = C64(input[2 * i], input[2 * i + 1]);
    const std::vector<C64> y = apply_sector_shift(s, t, terms, x);
    for (size_t i = 0; i < y.size(); ++i) {
      output[2 * i] = y[i].real();
      output[2 * i + 1] = y[i].imag();
    }
  });
}

// spectral_function (src/dynamics/mod.rs:964-1021) of the probed vector.
int oracle_spectral_function(void* target, const double* created, long long n_frequencies, const double* frequencies,
                             double reference_energy, double broadening, long long krylov, double tolerance,
                             double* out) {
  return guarded([&] {
    const Operator& op = *static_cast<Operator*>(target);
    std::vector<C64> v(op.rows);
    for (size_t i = 0; i < op.rows; ++i) v[i] = C64(created[2 * i], created[2 * i + 1]);
    const std::vector<double> f(frequencies, frequencies + std::max(n_frequencies, 0LL));
    const std::vector<double> r = spectral_function(op, v, f, reference_energy, broadening,
                                                    static_cast<size_t>(std::max(krylov, 0LL)), tolerance);
    for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
  });
}

}  // extern "C"
