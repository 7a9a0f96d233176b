// Matrix-free H.v and block action on u64 states: flip programs, image tables
// and the warp-tile kernel (see hv_tile.cuh).
//
// Reference behaviour (matrixlab-research/QMBED):
//   visit_unreduced_local_transitions_with_symbols  src/basis/mod.rs:1122-1232
//   index_transition (sqrt(R_src/R_tgt) conj(phase))  src/basis/mod.rs:1561-1580
//   fixed_weight_state_index (colex rank)            src/basis/mod.rs:640-659
//   spin_symmetry_sector (orbit minimum, characters) src/basis/mod.rs:715-848
//   apply / apply_real                                src/operator/mod.rs:1414-1548
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "device_util.cuh"
#include "hv_tile.cuh"
#include "operator.cuh"

namespace qmbed {

namespace {

constexpr int kRankChunkBits = 4;
constexpr int kRankChunkValues = 1 << kRankChunkBits;
constexpr size_t kRankTableMaxBytes = 40 * 1024;
constexpr int kMaxFences = 4096;
constexpr size_t kProgramSmemMax = 32 * 1024;
constexpr int kTileThreads = 256;
constexpr uint64_t kAllOnes = ~0ull;

using TermKey = std::tuple<uint64_t, uint64_t, uint64_t>;  // req_mask, req_val, sign_mask

// Amplitude of one term on the state whose bits at sites i, j are (v & 1, v >> 1).
double term_sign(const TermKey& key, int i, int j, int v, bool* allowed) {
  const auto& [req_mask, req_val, sign_mask] = key;
  auto bit_of = [&](int site) -> uint64_t {
    if (site == i) return static_cast<uint64_t>(v & 1);
    return static_cast<uint64_t>((v >> 1) & 1);
  };
  uint64_t state = 0;
  for (int site : {i, j}) state |= bit_of(site) << site;
  *allowed = (state & req_mask) == req_val;
  const int zeros = __builtin_popcountll(~state & sign_mask & ((1ull << i) | (1ull << j)));
  return (zeros & 1) ? -1.0 : 1.0;
}

// Sites (i <= j) carrying every bit of `u`, when u has at most two bits.
bool two_sites(uint64_t u, int* i, int* j) {
  const int n = __builtin_popcountll(u);
  if (n > 2) return false;
  if (n == 0) {
    *i = *j = 0;
    return true;
  }
  *i = __builtin_ctzll(u);
  *j = 63 - __builtin_clzll(u);
  return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// Flip programs (host)
// ---------------------------------------------------------------------------

namespace {

// Chain classes from pair tables: bond (i, i + d mod L), digits v = d_i | d_{i+d} << 1.
struct ChainBuilder {
  int sites;
  bool ok = true;
  std::vector<ChainClass> classes;

  void add(int a, int b, const double* re, const double* im, int nz) {
    // a < b: orient the bond as (i, i + d) with d <= L / 2
    int i = a, d = b - a;
    bool swap = false;
    if (d > sites - d) {
      i = b;
      d = sites - d;
      swap = true;  // the table's first digit is then the bond's second site
    }
    double r[4], m[4];
    int z = 0;
    for (int v = 0; v < 4; ++v) {
      const int w = swap ? (((v & 1) << 1) | (v >> 1)) : v;
      r[v] = re[w];
      m[v] = im[w];
      if ((nz >> w) & 1) z |= 1 << v;
    }
    for (ChainClass& c : classes) {
      if (c.d != d) continue;
      if (c.nz != z || std::memcmp(c.re, r, sizeof r) != 0 || std::memcmp(c.im, m, sizeof m) != 0) ok = false;
      if (c.bonds & (1ull << i)) ok = false;
      c.bonds |= 1ull << i;
      return;
    }
    ChainClass c{};
    c.bonds = 1ull << i;
    c.d = d;
    c.nz = z;
    std::memcpy(c.re, r, sizeof r);
    std::memcpy(c.im, m, sizeof m);
    classes.push_back(c);
  }
};

}  // namespace

FlipProgram compile_flip_program(const std::vector<Instance>& adjoint, const LocalFactors& f, int sites,
                                 bool fixed_weight) {
  FlipProgram prog;
  if (sites > 64) return prog;
  // spin-1/2 factors: z(d) = z1 * (+1 | -1), ladder factors independent of d
  if (f.z[0] != -f.z[1] || f.raise != f.lower) return prog;
  std::map<uint64_t, std::map<TermKey, C64>> by_flip;
  for (const Instance& a : adjoint) {
    uint64_t seen = 0, flip = 0, req_mask = 0, req_val = 0, sign_mask = 0;
    C64 k(a.cr, a.ci);
    for (int q = 0; q < a.n; ++q) {
      const char sym = a.sym[q];
      if (sym == 'I') continue;
      const uint64_t bit = 1ull << a.site[q];
      if (seen & bit) return FlipProgram{};  // a repeated site: the digit changes between factors
      seen |= bit;
      switch (sym) {
        case 'z':
          sign_mask |= bit;
          k *= f.z[1];
          break;
        case '+':
          flip |= bit;
          req_mask |= bit;
          k *= f.raise;
          break;
        case '-':
          flip |= bit;
          req_mask |= bit;
          req_val |= bit;
          k *= f.lower;
          break;
        case 'x':
          flip |= bit;
          k *= f.xy_scale * f.raise;
          break;
        case 'y':
          // (d ? +i : -i) * g: i g times the sign of the digit
          flip |= bit;
          sign_mask |= bit;
          k *= C64(0.0, f.xy_scale * f.raise);
          break;
        default:
          return FlipProgram{};
      }
    }
    if (k == C64(0.0, 0.0)) continue;
    // the row entry is conj(coefficient * amplitude)
    by_flip[flip][{req_mask, req_val, sign_mask}] += std::conj(k);
  }
  // Products whose amplitude depends on at most two sites (those they flip
  // included) become 4-entry amplitude tables indexed by the two digits.
  auto add_slot = [&](const std::map<TermKey, C64>& terms, int i, int j, uint8_t* nz) {
    C64 amp[4];
    for (int v = 0; v < 4; ++v)
      for (const auto& [key, k] : terms) {
        bool allowed = false;
        const double sign = term_sign(key, i, j, v, &allowed);
        if (allowed) amp[v] += sign * k;
      }
    *nz = 0;
    for (int v = 0; v < 4; ++v) {
      prog.amp_re.push_back(amp[v].real());
      prog.amp_im.push_back(amp[v].imag());
      if (amp[v].imag() != 0.0) prog.complex_coefs = true;
      if (amp[v] != C64(0.0, 0.0)) *nz |= static_cast<uint8_t>(1u << v);
    }
  };
  // diagonal products: grouped by the (at most two) sites they read
  if (by_flip.count(0)) {
    std::map<std::pair<int, int>, std::map<TermKey, C64>> pairs;
    for (const auto& [key, k] : by_flip[0]) {
      if (k == C64(0.0, 0.0)) continue;
      int i = 0, j = 0;
      if (two_sites(std::get<0>(key) | std::get<2>(key), &i, &j)) {
        pairs[{i, j}][key] += k;
      } else {
        FlipTerm t{std::get<0>(key), std::get<1>(key), std::get<2>(key), k.real(), k.imag()};
        if (t.ki != 0.0) prog.complex_coefs = true;
        prog.diag_terms.push_back(t);
      }
    }
    for (const auto& [sites_ij, terms] : pairs) {
      uint8_t nz = 0;
      add_slot(terms, sites_ij.first, sites_ij.second, &nz);
      prog.diag_pairs.push_back(static_cast<uint32_t>(sites_ij.first) | (static_cast<uint32_t>(sites_ij.second) << 8));
    }
  }
  for (const auto& [flip, terms] : by_flip) {
    if (flip == 0) continue;
    std::map<TermKey, C64> live;
    uint64_t reads = flip;
    for (const auto& [key, k] : terms)
      if (k != C64(0.0, 0.0)) {
        live[key] = k;
        reads |= std::get<0>(key) | std::get<2>(key);
      }
    if (live.empty()) continue;
    FlipGroup g{};
    g.flip = flip;
    g.chunk_lo = static_cast<uint8_t>(__builtin_ctzll(flip) / 4);
    g.chunk_hi = static_cast<uint8_t>((63 - __builtin_clzll(flip)) / 4);
    int i = 0, j = 0;
    if (two_sites(reads, &i, &j)) {
      g.kind = kGroupPair;
      g.site_i = static_cast<uint8_t>(i);
      g.site_j = static_cast<uint8_t>(j);
      g.first = static_cast<uint32_t>(prog.amp_re.size() / 4);
      add_slot(live, i, j, &g.nz);
      if (fixed_weight) {
        // a flip keeps the weight only when it moves one up spin: two flipped
        // sites with different digits (v = 1, 2)
        g.nz &= (__builtin_popcountll(flip) == 2) ? 0x6 : 0x0;
      }
      if (g.nz == 0) {  // every amplitude cancels, or every target leaves the space
        prog.amp_re.resize(prog.amp_re.size() - 4);
        prog.amp_im.resize(prog.amp_im.size() - 4);
        continue;
      }
    } else {
      g.kind = kGroupGeneric;
      g.first = static_cast<uint32_t>(prog.terms.size());
      for (const auto& [key, k] : live) {
        FlipTerm t{std::get<0>(key), std::get<1>(key), std::get<2>(key), k.real(), k.imag()};
        if (t.ki != 0.0) prog.complex_coefs = true;
        prog.terms.push_back(t);
      }
      g.count = static_cast<uint16_t>(prog.terms.size() - g.first);
    }
    prog.groups.push_back(g);
  }
  prog.ok = true;
  // Translation-structured form: every group a two-site flip, every diagonal
  // part a site pair or a uniform single-site field, uniform per displacement.
  ChainBuilder off{sites}, diag{sites};
  bool chain = prog.terms.empty() && prog.diag_terms.empty();
  for (const FlipGroup& g : prog.groups) {
    if (!chain) break;
    if (g.kind != kGroupPair || g.site_i == g.site_j) {
      chain = false;
      break;
    }
    off.add(g.site_i, g.site_j, &prog.amp_re[4 * g.first], &prog.amp_im[4 * g.first], g.nz);
  }
  ChainProgram cp{};
  for (size_t q = 0; q < prog.diag_pairs.size() && chain; ++q) {
    const int i = prog.diag_pairs[q] & 0xff, j = prog.diag_pairs[q] >> 8;
    const double* re = &prog.amp_re[4 * q];
    const double* im = &prog.amp_im[4 * q];
    if (i != j) {
      diag.add(i, j, re, im, 0xf);
      continue;
    }
    // one site: digits 0 and 1 sit at v = 0 and v = 3
    if (cp.has_field && (cp.field_re[0] != re[0] || cp.field_re[1] != re[3] || cp.field_im[0] != im[0] ||
                         cp.field_im[1] != im[3] || (cp.field_mask & (1ull << i)))) {
      chain = false;
      break;
    }
    cp.has_field = 1;
    cp.field_mask |= 1ull << i;
    cp.field_re[0] = re[0];
    cp.field_re[1] = re[3];
    cp.field_im[0] = im[0];
    cp.field_im[1] = im[3];
  }
  chain = chain && off.ok && diag.ok && off.classes.size() <= static_cast<size_t>(kChainMaxOff) &&
          diag.classes.size() <= static_cast<size_t>(kChainMaxDiag);
  if (chain) {
    cp.n_off = static_cast<int>(off.classes.size());
    cp.n_diag = static_cast<int>(diag.classes.size());
    for (int c = 0; c < cp.n_off; ++c) cp.off[c] = off.classes[static_cast<size_t>(c)];
    for (int c = 0; c < cp.n_diag; ++c) cp.diag[c] = diag.classes[static_cast<size_t>(c)];
    prog.chain = cp;
    prog.chain_ok = true;
  }
  return prog;
}

void DeviceFlipProgram::upload(const FlipProgram& prog) {
  ok_ = prog.ok;
  if (!ok_) return;
  complex_ = prog.complex_coefs;
  chain_ok_ = prog.chain_ok;
  chain_ = prog.chain;
  n_dterms_ = static_cast<int>(prog.diag_terms.size());
  n_terms_ = n_dterms_ + static_cast<int>(prog.terms.size());
  n_groups_ = static_cast<int>(prog.groups.size());
  n_slots_ = static_cast<int>(prog.amp_re.size() / 4);
  n_dpairs_ = static_cast<int>(prog.diag_pairs.size());
  std::vector<FlipTerm> all(prog.diag_terms);
  all.insert(all.end(), prog.terms.begin(), prog.terms.end());
  // generic group terms follow the generic diagonal terms
  std::vector<FlipGroup> groups(prog.groups);
  for (FlipGroup& g : groups)
    if (g.kind == kGroupGeneric) g.first += static_cast<uint32_t>(n_dterms_);
  // [terms][groups][amp_re][amp_im][diag pair sites], every part 8-byte aligned
  groups_offset_ = all.size() * sizeof(FlipTerm);
  amp_offset_ = groups_offset_ + groups.size() * sizeof(FlipGroup);
  pairs_offset_ = amp_offset_ + 2 * prog.amp_re.size() * sizeof(double);
  bytes_ = pairs_offset_ + ((prog.diag_pairs.size() + 1) / 2) * 8;
  std::vector<char> host(std::max<size_t>(bytes_, 16), 0);
  if (!all.empty()) std::memcpy(host.data(), all.data(), groups_offset_);
  if (!groups.empty()) std::memcpy(host.data() + groups_offset_, groups.data(), groups.size() * sizeof(FlipGroup));
  if (!prog.amp_re.empty()) {
    std::memcpy(host.data() + amp_offset_, prog.amp_re.data(), prog.amp_re.size() * sizeof(double));
    std::memcpy(host.data() + amp_offset_ + prog.amp_re.size() * sizeof(double), prog.amp_im.data(),
                prog.amp_im.size() * sizeof(double));
  }
  if (!prog.diag_pairs.empty())
    std::memcpy(host.data() + pairs_offset_, prog.diag_pairs.data(), prog.diag_pairs.size() * sizeof(uint32_t));
  buf_.allocate(host.size());
  QMBED_CUDA(cudaMemcpy(buf_.get(), host.data(), host.size(), cudaMemcpyHostToDevice));
}

namespace {

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Colex rank from 4-bit chunk tables: tab[(c * 16 + v) * stride + k] is the
// rank contribution of the set bits v of chunk c when k set bits lie below
// it (fixed_weight_state_index, src/basis/mod.rs:640-659, summed per chunk).
// The set bits below each chunk come from a masked popcount, so the chunk
// reads do not wait on one another.
__device__ __forceinline__ uint64_t rank_chunked(uint64_t t, const uint64_t* __restrict__ tab, int chunks,
                                                 int stride) {
  uint64_t r = 0;
#pragma unroll 4
  for (int c = 0; c < chunks; ++c) {
    const unsigned v = static_cast<unsigned>(t >> (kRankChunkBits * c)) & (kRankChunkValues - 1);
    const int ones = __popcll(t & ((1ull << (kRankChunkBits * c)) - 1));
    r += tab[(c * kRankChunkValues + v) * stride + ones];
  }
  return r;
}

// Rank of t = s ^ flip from the rank of s when both have the same weight:
// only chunks lo..hi (those holding flipped bits, and the ones between them)
// change their contribution.
__device__ __forceinline__ uint64_t rank_delta(uint64_t s, uint64_t t, uint64_t rank_s, int lo, int hi,
                                               const uint64_t* __restrict__ tab, int stride) {
  uint64_t r = rank_s;
  const uint64_t below = (1ull << (kRankChunkBits * lo)) - 1;
  int ones_s = __popcll(s & below), ones_t = ones_s;
  for (int c = lo; c <= hi; ++c) {
    const unsigned vs = static_cast<unsigned>(s >> (kRankChunkBits * c)) & (kRankChunkValues - 1);
    const unsigned vt = static_cast<unsigned>(t >> (kRankChunkBits * c)) & (kRankChunkValues - 1);
    r += tab[(c * kRankChunkValues + vt) * stride + ones_t] - tab[(c * kRankChunkValues + vs) * stride + ones_s];
    ones_s += __popc(vs);
    ones_t += __popc(vt);
  }
  return r;
}

__device__ __forceinline__ int digit_pair(uint64_t s, uint32_t i, uint32_t j) {
  return static_cast<int>((s >> i) & 1) | (static_cast<int>((s >> j) & 1) << 1);
}

struct TileArgs {
  SectorParams p;
  uint64_t mask;
  uint64_t dim;
  uint64_t row0, rows;  // rows computed: row0 .. row0 + rows - 1 (outputs indexed from row0)
  const uint64_t* states;
  const uint16_t* orbits;
  // program (copied to shared memory by every block)
  const unsigned long long* program;
  int program_words;
  int n_dterms, n_terms, n_groups, n_slots, n_dpairs;
  int groups_offset, amp_offset, pairs_offset;  // bytes
  // lookups
  const uint64_t* rank_tab;  // chunk tables (shared memory copy in the kernel)
  int rank_chunks, rank_stride;
  const uint64_t* binom;
  const void* table;
  int table_wide;
  int idx_bits, rbits, mbits;
  const double* class_inv_sqrt;  // orbit class -> 1/sqrt(R)
  const double* phase_m;         // m -> exp(-2 pi i m / L)
  const double* phase_shift;     // shift -> character of the basis phase table
  const double* inv_sqrt;        // [R] 1/sqrt(R), [257 + R] sqrt(R)
  const uint64_t* fences;
  int n_fences;
  uint64_t fence_seg;
  int fence_levels;  // iterations of the global search inside one segment
  // vectors
  const void* x;
  const void* pv;
  void* y;
  double alpha, beta, gamma;
  ChainProgram chain;
  int binom_rows;  // chain path: C(n, k), n < binom_rows, k <= up, staged in shared memory
};

enum TileMode : int { kModeDirect = 0, kModeColex = 1, kModeTable = 2, kModeSearch = 3 };

// Shared-memory view of a flip program.
struct Program {
  const FlipTerm* terms;
  const FlipGroup* groups;
  const double* amp_re;
  const double* amp_im;
  const uint32_t* pairs;
};

// Sum over generic terms [first, first + count) of [s & req == val] k (-1)^popc(~s & sign).
template <bool CPLX>
__device__ __forceinline__ void terms_amplitude(const FlipTerm* __restrict__ terms, uint32_t first, uint32_t count,
                                                uint64_t s, double& ar, double& ai) {
  for (uint32_t i = first; i < first + count; ++i) {
    const FlipTerm& t = terms[i];
    if ((s & t.req_mask) != t.req_val) continue;
    const bool neg = __popcll(~s & t.sign_mask) & 1;
    ar += neg ? -t.kr : t.kr;
    if (CPLX) ai += neg ? -t.ki : t.ki;
  }
}

template <bool CPLX>
__device__ __forceinline__ void group_amplitude(const Program& pg, const FlipGroup& g, uint64_t s, double& ar,
                                                double& ai) {
  ar = 0.0;
  ai = 0.0;
  if (g.kind == kGroupPair) {
    const int v = digit_pair(s, g.site_i, g.site_j);
    ar = pg.amp_re[4 * g.first + v];
    if (CPLX) ai = pg.amp_im[4 * g.first + v];
  } else {
    terms_amplitude<CPLX>(pg.terms, g.first, g.count, s, ar, ai);
  }
}

__device__ __forceinline__ bool group_active(const Program& pg, const FlipGroup& g, uint64_t s) {
  if (g.kind == kGroupPair) return (g.nz >> digit_pair(s, g.site_i, g.site_j)) & 1;
  bool any = false;
  for (uint32_t i = g.first; i < g.first + g.count; ++i) any |= (s & pg.terms[i].req_mask) == pg.terms[i].req_val;
  return any;
}

// Per-target lookup result: column (-1: not in the basis), character
// (chi_r, chi_i) and 1/sqrt(R_column) (1 without symmetry).
struct Hit {
  int64_t col;
  double cr, ci;
  double inv_sqrt_rc;
};

// Rank of target t (same weight as the row state s): incremental over the
// chunks the flip touches when they are few, else from scratch.
__device__ __forceinline__ uint64_t target_rank(const TileArgs& a, const uint64_t* __restrict__ s_rank, uint64_t s,
                                                uint64_t t, uint64_t rank_s, int lo, int hi) {
  return hi - lo <= 2 ? rank_delta(s, t, rank_s, lo, hi, s_rank, a.rank_stride)
                      : rank_chunked(t, s_rank, a.rank_chunks, a.rank_stride);
}

template <int U, int MODE, bool NEED_R>
__device__ __forceinline__ void lookup_batch(const TileArgs& a, const uint64_t* __restrict__ s_rank,
                                             const uint64_t* __restrict__ s_fence, uint64_t s, uint64_t rank_s,
                                             const bool (&act)[U], const uint64_t (&t)[U], const int (&lo)[U],
                                             const int (&hi)[U], const uint64_t (&rank_t)[U], Hit (&h)[U]) {
#pragma unroll
  for (int u = 0; u < U; ++u) h[u] = Hit{-1, 1.0, 0.0, 1.0};
  if (MODE == kModeDirect) {
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (act[u] && t[u] < a.dim) h[u].col = static_cast<int64_t>(t[u]);
  } else if (MODE == kModeColex) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!act[u] || __popcll(t[u]) != a.p.up) continue;
      if (rank_t[u] != kAllOnes) h[u].col = static_cast<int64_t>(rank_t[u]);
      else h[u].col = a.rank_chunks > 0 ? static_cast<int64_t>(target_rank(a, s_rank, s, t[u], rank_s, lo[u], hi[u]))
                                        : colex_rank_checked(t[u], a.p.sites, a.p.up, a.binom);
    }
  } else if (MODE == kModeTable) {
    uint64_t e[U];
    // ranks first, then all table reads, so the reads are in flight together
#pragma unroll
    for (int u = 0; u < U; ++u) {
      e[u] = kAllOnes;
      if (!act[u]) continue;
      if (a.p.up >= 0 && rank_t[u] == kAllOnes && __popcll(t[u]) != a.p.up) continue;
      const uint64_t rank = a.p.up < 0 ? t[u]
                            : rank_t[u] != kAllOnes ? rank_t[u]
                                                    : target_rank(a, s_rank, s, t[u], rank_s, lo[u], hi[u]);
      if (a.table_wide) {
        e[u] = __ldg(static_cast<const unsigned long long*>(a.table) + rank);
      } else {
        const uint32_t v = __ldg(static_cast<const uint32_t*>(a.table) + rank);
        e[u] = v == 0xffffffffu ? kAllOnes : v;
      }
    }
    const uint64_t idx_mask = (1ull << a.idx_bits) - 1;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (e[u] == kAllOnes) continue;
      const uint64_t code = e[u] >> a.idx_bits;
      h[u].col = static_cast<int64_t>(e[u] & idx_mask);
      const bool neg = code & 1;
      if (a.mbits > 0) {
        const int m = static_cast<int>(code >> (1 + a.rbits));
        h[u].cr = __ldg(a.phase_m + 2 * m);
        h[u].ci = __ldg(a.phase_m + 2 * m + 1);
      }
      if (neg) {
        h[u].cr = -h[u].cr;
        h[u].ci = -h[u].ci;
      }
      if (NEED_R) h[u].inv_sqrt_rc = __ldg(a.class_inv_sqrt + ((code >> 1) & ((1u << a.rbits) - 1)));
    }
  } else {  // kModeSearch
    uint64_t key[U];
    int shift[U];
    bool neg[U];
    uint32_t fb[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      key[u] = 0;
      shift[u] = 0;
      neg[u] = false;
      fb[u] = 0;
      if (!act[u]) continue;
      const Canonical<uint64_t> c = canonicalize(t[u], a.p, a.mask);
      key[u] = c.rep;
      shift[u] = c.shift;
      neg[u] = (c.reflected && a.p.parity < 0) != (c.inverted && a.p.inversion < 0);
    }
    // fence keys in shared memory: the segment that can hold each key
    for (int len = a.n_fences; len > 1;) {
      const int half = len >> 1;
#pragma unroll
      for (int u = 0; u < U; ++u) fb[u] = (s_fence[fb[u] + half] <= key[u]) ? fb[u] + half : fb[u];
      len -= half;
    }
    uint64_t base[U], len[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      base[u] = static_cast<uint64_t>(fb[u]) * a.fence_seg;
      len[u] = min(a.fence_seg, a.dim - base[u]);
    }
    for (int it = 0; it < a.fence_levels; ++it) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (len[u] <= 1) continue;
        const uint64_t half = len[u] >> 1;
        base[u] = (__ldg(a.states + base[u] + half) <= key[u]) ? base[u] + half : base[u];
        len[u] -= half;
      }
    }
    uint64_t found[U];
#pragma unroll
    for (int u = 0; u < U; ++u) found[u] = act[u] ? __ldg(a.states + base[u]) : ~key[u];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!act[u] || found[u] != key[u]) continue;
      h[u].col = static_cast<int64_t>(base[u]);
      h[u].cr = __ldg(a.phase_shift + 2 * shift[u]);
      h[u].ci = __ldg(a.phase_shift + 2 * shift[u] + 1);
      if (neg[u]) {
        h[u].cr = -h[u].cr;
        h[u].ci = -h[u].ci;
      }
    }
    if (NEED_R) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (h[u].col >= 0) h[u].inv_sqrt_rc = __ldg(a.inv_sqrt + __ldg(a.orbits + h[u].col));
    }
  }
}

// Targets per lane per round: U lookups (and gathers) in flight per lane.
template <typename T, int NB, bool CPLX>
struct TileShape {
  static constexpr int U = NB == 1 ? 4 : (NB * sizeof(T) <= 32 ? 4 : (NB * sizeof(T) <= 64 ? 2 : 1));
  static constexpr int MIN_BLOCKS = (NB == 1 || NB * sizeof(T) <= 32) ? 3 : 2;
};

// Resolves a round of U targets and accumulates their contributions:
// acc += w chi / sqrt(R_c) x[c] (NB = 1) or acc[:] += w chi z[c][:] (blocks).
template <typename T, int NB, bool CPLX, int MODE, int U>
__device__ __forceinline__ void consume_round(const TileArgs& a, const uint64_t* __restrict__ s_rank,
                                              const uint64_t* __restrict__ s_fence, uint64_t s, uint64_t rank_s,
                                              const bool (&act)[U], const uint64_t (&t)[U], const int (&lo)[U],
                                              const int (&hi)[U], const double (&wr)[U], const double (&wi)[U],
                                              const T* __restrict__ x, T (&acc)[NB], T& acc_i,
                                              const uint64_t (&rank_t)[U]) {
  constexpr bool NEED_R = NB == 1;
  constexpr int VEC = 16 / sizeof(T);
  constexpr int PARTS = NB >= VEC ? NB / VEC : 1;
  Hit h[U];
  lookup_batch<U, MODE, NEED_R>(a, s_rank, s_fence, s, rank_s, act, t, lo, hi, rank_t, h);
  if (NB == 1) {
    T gr[U], gi[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      gr[u] = 0;
      gi[u] = 0;
      if (h[u].col < 0) continue;
      if (CPLX) {
        gr[u] = __ldg(x + 2 * h[u].col);
        gi[u] = __ldg(x + 2 * h[u].col + 1);
      } else {
        gr[u] = __ldg(x + h[u].col);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (h[u].col < 0) continue;
      if (CPLX) {
        // w * chi / sqrt(R_c)
        const double fr = (wr[u] * h[u].cr - wi[u] * h[u].ci) * h[u].inv_sqrt_rc;
        const double fi = (wr[u] * h[u].ci + wi[u] * h[u].cr) * h[u].inv_sqrt_rc;
        acc[0] += static_cast<T>(fr) * gr[u] - static_cast<T>(fi) * gi[u];
        acc_i += static_cast<T>(fr) * gi[u] + static_cast<T>(fi) * gr[u];
      } else {
        // real operators: chi = +-1
        acc[0] += static_cast<T>(wr[u] * h[u].cr * h[u].inv_sqrt_rc) * gr[u];
      }
    }
  } else {
    T g[U][NB];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (h[u].col < 0) {
#pragma unroll
        for (int j = 0; j < NB; ++j) g[u][j] = 0;
        continue;
      }
      const T* row = x + static_cast<uint64_t>(h[u].col) * NB;
#pragma unroll
      for (int q = 0; q < PARTS; ++q) {
        T v[VEC];
        load16(row + q * VEC, v);
#pragma unroll
        for (int j = 0; j < VEC; ++j) g[u][q * VEC + j] = v[j];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      // real operators: the entry is w * chi, chi = +-1
      const T c = h[u].col < 0 ? static_cast<T>(0) : static_cast<T>(wr[u] * h[u].cr);
#pragma unroll
      for (int j = 0; j < NB; ++j) acc[j] += c * g[u][j];
    }
  }
}

// State rotated so that bit i holds digit (i + d) mod L.
__device__ __forceinline__ uint64_t digits_ahead(uint64_t s, int d, int sites, uint64_t mask) {
  return ((s >> d) | (s << (sites - d))) & mask;
}

// One warp per tile of 32 consecutive rows, one lane per row. Each lane
// marks its row's active transitions in a bit mask; the warp then pops U of
// them per lane per round, so every lane stays busy until the row with the
// most transitions in the tile is done. CHAIN programs take their masks and
// diagonal from word operations per bond class; others visit their groups.
// NB = 1 computes y = H x (orbit ratio sqrt(R_r / R_c) applied, x real or
// interleaved complex); NB = 8/16 computes the block action in orbit-scaled
// coordinates with the three-term epilogue.
template <typename T, int NB, bool CPLX, int MODE, bool HAS_P, bool CHAIN>
__global__ void __launch_bounds__(kTileThreads, TileShape<T, NB, CPLX>::MIN_BLOCKS)
    hv_tile_kernel(const __grid_constant__ TileArgs a) {
  constexpr int U = TileShape<T, NB, CPLX>::U;
  constexpr int VEC = 16 / sizeof(T);
  constexpr int PARTS = NB >= VEC ? NB / VEC : 1;
  constexpr bool RANKED = MODE == kModeColex || MODE == kModeTable;
  extern __shared__ __align__(16) unsigned char smem[];
  // shared memory: [flip program][rank chunk table][fence keys]
  unsigned long long* words = reinterpret_cast<unsigned long long*>(smem);
  for (int i = threadIdx.x; i < a.program_words; i += blockDim.x) words[i] = a.program[i];
  const size_t rank_words =
      RANKED && a.rank_chunks > 0 ? static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride : 0;
  uint64_t* s_rank = reinterpret_cast<uint64_t*>(words + a.program_words);
  for (size_t i = threadIdx.x; i < rank_words; i += blockDim.x) s_rank[i] = a.rank_tab[i];
  uint64_t* s_fence = s_rank + rank_words;
  if (MODE == kModeSearch)
    for (int i = threadIdx.x; i < a.n_fences; i += blockDim.x) s_fence[i] = a.fences[i];
  // chain path of ranked lookups: binomials for the nearest-neighbour rank step
  uint64_t* s_binom = s_fence + (MODE == kModeSearch ? a.n_fences : 0);
  const int binom_stride = a.p.up + 1;
  if (CHAIN && RANKED)
    for (int i = threadIdx.x; i < a.binom_rows * binom_stride; i += blockDim.x)
      s_binom[i] = a.binom[(i / binom_stride) * kBinomStride + i % binom_stride];
  __syncthreads();
  Program pg;
  pg.terms = reinterpret_cast<const FlipTerm*>(smem);
  pg.groups = reinterpret_cast<const FlipGroup*>(smem + a.groups_offset);
  pg.amp_re = reinterpret_cast<const double*>(smem + a.amp_offset);
  pg.amp_im = pg.amp_re + 4 * a.n_slots;
  pg.pairs = reinterpret_cast<const uint32_t*>(smem + a.pairs_offset);

  const int lane = threadIdx.x & 31;
  const int L = a.p.sites;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const T* x = static_cast<const T*>(a.x);
  const bool ranked_rows = RANKED && a.p.up >= 0 && a.rank_chunks > 0;
  for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 32 < a.rows;
       tile += warps) {
    // row r of the operator; `slot` indexes the outputs (rows row0 .. row0 + rows - 1)
    const uint64_t slot = tile * 32 + lane;
    const uint64_t r = a.row0 + slot;
    const bool valid = slot < a.rows;
    uint64_t s = 0;
    if (valid) s = MODE == kModeDirect ? r : __ldcs(a.states + r);
    const uint64_t rank_s = ranked_rows ? rank_chunked(s, s_rank, a.rank_chunks, a.rank_stride) : 0;
    double dr = 0.0, di = 0.0;
    T acc[NB], acc_i = 0;
#pragma unroll
    for (int j = 0; j < NB; ++j) acc[j] = 0;
    if (CHAIN) {
      const ChainProgram& ch = a.chain;
      if (valid) {
        if (ch.has_field) {
          const int ones = __popcll(s & ch.field_mask), zeros = __popcll(~s & ch.field_mask);
          dr += zeros * ch.field_re[0] + ones * ch.field_re[1];
          if (CPLX) di += zeros * ch.field_im[0] + ones * ch.field_im[1];
        }
        for (int c = 0; c < ch.n_diag; ++c) {
          const ChainClass& cl = ch.diag[c];
          const uint64_t b = digits_ahead(s, cl.d, L, a.mask);
          const int n[4] = {__popcll(~s & ~b & cl.bonds), __popcll(s & ~b & cl.bonds), __popcll(~s & b & cl.bonds),
                            __popcll(s & b & cl.bonds)};
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            dr += n[v] * cl.re[v];
            if (CPLX) di += n[v] * cl.im[v];
          }
        }
      }
      for (int c = 0; c < ch.n_off; ++c) {
        const ChainClass& cl = ch.off[c];
        const uint64_t b = digits_ahead(s, cl.d, L, a.mask);
        uint64_t active = 0;
        if (valid) {
          if (cl.nz & 1) active |= ~s & ~b;
          if (cl.nz & 2) active |= s & ~b;
          if (cl.nz & 4) active |= ~s & b;
          if (cl.nz & 8) active |= s & b;
          active &= cl.bonds;
        }
        while (__any_sync(0xffffffffu, active != 0)) {
          bool act[U];
          uint64_t t[U];
          int lo[U], hi[U];
          double wr[U], wi[U];
          uint64_t rank_t[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            act[u] = active != 0;
            t[u] = 0;
            lo[u] = 0;
            hi[u] = 0;
            wr[u] = 0.0;
            wi[u] = 0.0;
            rank_t[u] = kAllOnes;
            if (!act[u]) continue;
            // the bond's first site as a one-bit mask, its partner d sites ahead
            const uint64_t first = active & (0ull - active);
            active ^= first;
            const uint64_t partner = ((first << cl.d) | (first >> (L - cl.d))) & a.mask;
            const bool d0 = (s & first) != 0, d1 = (s & partner) != 0;
            const int v = (d0 ? 1 : 0) | (d1 ? 2 : 0);
            wr[u] = cl.re[v];
            if (CPLX) wi[u] = cl.im[v];
            t[u] = s ^ first ^ partner;
            const uint64_t below = first - 1;
            const int i = __popcll(below);
            const int j = partner > first ? i + cl.d : i + cl.d - L;
            lo[u] = min(i, j) >> 2;
            hi[u] = max(i, j) >> 2;
            if (RANKED && ranked_rows && cl.d == 1 && partner > first) {
              // one up spin hops between neighbours i, i+1 with k up spins below:
              // the colex rank moves by C(i, k) (up) or -C(i, k) (down)
              const uint64_t step = s_binom[i * binom_stride + __popcll(s & below)];
              rank_t[u] = d0 ? rank_s + step : rank_s - step;
            }
          }
          consume_round<T, NB, CPLX, MODE, U>(a, s_rank, s_fence, s, rank_s, act, t, lo, hi, wr, wi, x, acc, acc_i,
                                              rank_t);
        }
      }
    } else {
      if (valid) {
        for (int q = 0; q < a.n_dpairs; ++q) {
          const uint32_t ij = pg.pairs[q];
          const int v = digit_pair(s, ij & 0xff, ij >> 8);
          dr += pg.amp_re[4 * q + v];
          if (CPLX) di += pg.amp_im[4 * q + v];
        }
        terms_amplitude<CPLX>(pg.terms, 0, a.n_dterms, s, dr, di);
      }
      for (int g0 = 0; g0 < a.n_groups; g0 += 64) {
        const int gn = min(64, a.n_groups - g0);
        uint64_t active = 0;
        if (valid)
          for (int g = 0; g < gn; ++g)
            if (group_active(pg, pg.groups[g0 + g], s)) active |= 1ull << g;
        while (__any_sync(0xffffffffu, active != 0)) {
          bool act[U];
          uint64_t t[U];
          int lo[U], hi[U];
          double wr[U], wi[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            act[u] = active != 0;
            t[u] = 0;
            lo[u] = 0;
            hi[u] = 0;
            wr[u] = 0.0;
            wi[u] = 0.0;
            if (!act[u]) continue;
            const int g = __ffsll(static_cast<long long>(active)) - 1;
            active &= active - 1;
            const FlipGroup& grp = pg.groups[g0 + g];
            group_amplitude<CPLX>(pg, grp, s, wr[u], wi[u]);
            t[u] = s ^ grp.flip;
            lo[u] = grp.chunk_lo;
            hi[u] = grp.chunk_hi;
          }
          uint64_t rank_t[U];
#pragma unroll
          for (int u = 0; u < U; ++u) rank_t[u] = kAllOnes;
          consume_round<T, NB, CPLX, MODE, U>(a, s_rank, s_fence, s, rank_s, act, t, lo, hi, wr, wi, x, acc, acc_i,
                                              rank_t);
        }
      }
    }
    if (!valid) continue;
    if (NB == 1) {
      const T scale = a.p.symmetric ? static_cast<T>(__ldg(a.inv_sqrt + 257 + __ldcs(a.orbits + r))) : static_cast<T>(1);
      T* y = static_cast<T*>(a.y);
      if (CPLX) {
        const T xr = __ldcs(x + 2 * r), xi = __ldcs(x + 2 * r + 1);
        const T d_r = static_cast<T>(dr), d_i = static_cast<T>(di);
        __stcs(y + 2 * slot, scale * acc[0] + d_r * xr - d_i * xi);
        __stcs(y + 2 * slot + 1, scale * acc_i + d_r * xi + d_i * xr);
      } else {
        __stcs(y + slot, scale * acc[0] + static_cast<T>(dr) * __ldcs(x + r));
      }
    } else {
      const T d = static_cast<T>(dr);
      const T al = static_cast<T>(a.alpha), be = static_cast<T>(a.beta), ga = static_cast<T>(a.gamma);
      T* out = static_cast<T*>(a.y);
      const T* pv = static_cast<const T*>(a.pv);
#pragma unroll
      for (int q = 0; q < PARTS; ++q) {
        T self[VEC], o[VEC];
        load16(x + r * NB + q * VEC, self);
#pragma unroll
        for (int j = 0; j < VEC; ++j) o[j] = al * (acc[q * VEC + j] + d * self[j]) + be * self[j];
        if (HAS_P) {
          T pq[VEC];
          load16_rw(pv + slot * NB + q * VEC, pq);
#pragma unroll
          for (int j = 0; j < VEC; ++j) o[j] += ga * pq[j];
        }
        store16(out + slot * NB + q * VEC, o);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Nearest-neighbour hop kernel
// ---------------------------------------------------------------------------

// Arguments of the hop kernel: a chain program whose only off-diagonal class
// is the nearest-neighbour bond (d = 1), on a real fixed-weight sector with a
// 32-bit image table (Heisenberg and XXZ chains in their k = 0, pi sectors).
struct HopArgs {
  uint64_t dim;
  uint64_t row0, rows;  // rows computed: row0 .. row0 + rows - 1 (outputs indexed from row0)
  int sites, up;
  const uint64_t* states;
  const uint16_t* orbits;
  const uint64_t* rank_tab;
  int rank_chunks, rank_stride;
  const uint64_t* binom;      // [n][k] with row stride kBinomStride
  const uint32_t* table;
  int idx_bits, rbits, n_classes;
  const double* class_inv_sqrt;  // orbit class -> 1/sqrt(R)
  const double* inv_sqrt;        // [257 + R] sqrt(R)
  uint64_t bonds_inner;          // bonds (i, i + 1) with i < L - 1
  int wrap;                      // bond (L - 1, 0) present
  double w_down, w_up;           // entries of the hops from digits (1, 0) and (0, 1) of a bond
  ChainProgram chain;            // diagonal classes and field
  const void* x;
  const void* pv;
  void* y;
  double alpha, beta, gamma;
};

constexpr int kHopMaxClasses = 64;

template <typename T, int NB>
struct HopShape {
  static constexpr int U = NB == 1 ? 4 : (NB * sizeof(T) <= 64 ? 4 : 2);
  static constexpr int MIN_BLOCKS = NB == 1 ? 4 : (NB * sizeof(T) <= 32 ? 3 : 2);
};

// One warp per tile of 32 consecutive rows, one lane per row. A bond
// (i, i + 1) with different digits moves one up spin between neighbours, so
// the target's colex rank is the row's rank +- C(i, k), k = up spins below
// site i (fixed_weight_state_index, src/basis/mod.rs:640-659): one shared-
// memory read per transition. The target's image-table entry gives its
// column, character sign and orbit class. The wrapping bond (L - 1, 0)
// renumbers every up spin, so its rank comes from the chunk tables in a step
// of its own after the inner bonds. Contributions (index_transition,
// src/basis/mod.rs:1561-1580, apply_real src/operator/mod.rs:1414-1485):
// NB = 1 accumulates w chi x[c] / sqrt(R_c) and scales by sqrt(R_r); blocks
// accumulate w chi z[c][:] in orbit-scaled coordinates with the three-term
// epilogue out = alpha (acc + d z_r) + beta z_r + gamma p_r.
template <typename T, int NB, bool HAS_P>
__global__ void __launch_bounds__(kTileThreads, HopShape<T, NB>::MIN_BLOCKS)
    hop_tile_kernel(const __grid_constant__ HopArgs a) {
  constexpr int U = HopShape<T, NB>::U;
  constexpr int VEC = 16 / sizeof(T);
  constexpr int PARTS = NB >= VEC ? NB / VEC : 1;
  extern __shared__ __align__(16) unsigned char smem[];
  // shared memory: [rank chunk table][binomials C(i, k), i < L, k <= up][1/sqrt(R) per class]
  uint64_t* s_rank = reinterpret_cast<uint64_t*>(smem);
  const int rank_words = a.rank_chunks * kRankChunkValues * a.rank_stride;
  for (int i = threadIdx.x; i < rank_words; i += blockDim.x) s_rank[i] = a.rank_tab[i];
  uint64_t* s_binom = s_rank + rank_words;
  const int bstride = a.up + 1;
  for (int i = threadIdx.x; i < a.sites * bstride; i += blockDim.x)
    s_binom[i] = a.binom[(i / bstride) * kBinomStride + i % bstride];
  T* s_cls = reinterpret_cast<T*>(s_binom + a.sites * bstride);
  for (int i = threadIdx.x; i < a.n_classes; i += blockDim.x) s_cls[i] = static_cast<T>(a.class_inv_sqrt[i]);
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int L = a.sites;
  const uint64_t idx_mask = (1ull << a.idx_bits) - 1;
  const uint32_t cls_mask = (1u << a.rbits) - 1;
  const int cls_shift = a.idx_bits + 1;
  const T w_down = static_cast<T>(a.w_down), w_up = static_cast<T>(a.w_up);
  const T* x = static_cast<const T*>(a.x);
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const uint64_t mask = L == 64 ? ~0ull : (1ull << L) - 1;

  // Adds the contributions of up to U targets whose table entries are e[u]
  // (0xffffffff: outside the sector) with hop amplitudes w[u].
  auto consume = [&](const uint32_t (&e)[U], const T (&w)[U], T (&acc)[NB]) {
    if (NB == 1) {
      T g[U];
#pragma unroll
      for (int u = 0; u < U; ++u) g[u] = e[u] != 0xffffffffu ? __ldg(x + (e[u] & idx_mask)) : static_cast<T>(0);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (e[u] == 0xffffffffu) continue;
        T f = w[u] * s_cls[(e[u] >> cls_shift) & cls_mask];
        if ((e[u] >> a.idx_bits) & 1) f = -f;
        acc[0] += f * g[u];
      }
    } else {
      T g[U][NB];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (e[u] == 0xffffffffu) {
#pragma unroll
          for (int j = 0; j < NB; ++j) g[u][j] = 0;
          continue;
        }
        const T* row = x + static_cast<uint64_t>(e[u] & idx_mask) * NB;
#pragma unroll
        for (int q = 0; q < PARTS; ++q) {
          T v[VEC];
          load16(row + q * VEC, v);
#pragma unroll
          for (int j = 0; j < VEC; ++j) g[u][q * VEC + j] = v[j];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        T c = e[u] == 0xffffffffu ? static_cast<T>(0) : w[u];
        if ((e[u] >> a.idx_bits) & 1) c = -c;
#pragma unroll
        for (int j = 0; j < NB; ++j) acc[j] += c * g[u][j];
      }
    }
  };

  for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 32 < a.rows;
       tile += warps) {
    // row r of the operator; `slot` indexes the outputs (rows row0 .. row0 + rows - 1)
    const uint64_t slot = tile * 32 + lane;
    const uint64_t r = a.row0 + slot;
    const bool valid = slot < a.rows;
    const uint64_t s = valid ? __ldcs(a.states + r) : 0;
    const uint64_t rank_s = rank_chunked(s, s_rank, a.rank_chunks, a.rank_stride);
    double dr = 0.0;
    const ChainProgram& ch = a.chain;
    if (valid) {
      if (ch.has_field) dr += __popcll(~s & ch.field_mask) * ch.field_re[0] + __popcll(s & ch.field_mask) * ch.field_re[1];
      for (int c = 0; c < ch.n_diag; ++c) {
        const ChainClass& cl = ch.diag[c];
        const uint64_t b = digits_ahead(s, cl.d, L, mask);
        dr += __popcll(~s & ~b & cl.bonds) * cl.re[0] + __popcll(s & ~b & cl.bonds) * cl.re[1] +
              __popcll(~s & b & cl.bonds) * cl.re[2] + __popcll(s & b & cl.bonds) * cl.re[3];
      }
    }
    T acc[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) acc[j] = 0;
    // bit i: digits of sites i and i + 1 differ (one up spin can hop)
    uint64_t hop = valid ? ((s ^ (s >> 1)) & a.bonds_inner) : 0;
    while (__any_sync(0xffffffffu, hop != 0)) {
      uint32_t e[U];
      T w[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        e[u] = 0xffffffffu;
        w[u] = 0;
        if (hop == 0) continue;
        const int i = __ffsll(static_cast<long long>(hop)) - 1;
        hop &= hop - 1;
        const uint64_t below = (1ull << i) - 1;
        const bool down = (s >> i) & 1;  // the up spin sits at i and moves to i + 1
        const uint64_t step = s_binom[i * bstride + __popcll(s & below)];
        const uint64_t rank_t = down ? rank_s + step : rank_s - step;
        w[u] = down ? w_down : w_up;
        e[u] = __ldg(a.table + rank_t);
      }
      consume(e, w, acc);
    }
    if (a.wrap) {
      // bond (L - 1, 0): digit L - 1 differs from digit 0
      const bool on = valid && (((s >> (L - 1)) ^ s) & 1);
      if (__any_sync(0xffffffffu, on)) {
        uint32_t e[U];
        T w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          e[u] = 0xffffffffu;
          w[u] = 0;
        }
        if (on) {
          const uint64_t t = s ^ (1ull << (L - 1)) ^ 1ull;
          const bool down = (s >> (L - 1)) & 1;
          w[0] = down ? w_down : w_up;
          e[0] = __ldg(a.table + rank_chunked(t, s_rank, a.rank_chunks, a.rank_stride));
        }
        consume(e, w, acc);
      }
    }
    if (!valid) continue;
    if (NB == 1) {
      const T scale = static_cast<T>(__ldg(a.inv_sqrt + 257 + __ldcs(a.orbits + r)));
      T* y = static_cast<T*>(a.y);
      __stcs(y + slot, scale * acc[0] + static_cast<T>(dr) * __ldcs(x + r));
    } else {
      const T d = static_cast<T>(dr);
      const T al = static_cast<T>(a.alpha), be = static_cast<T>(a.beta), ga = static_cast<T>(a.gamma);
      T* out = static_cast<T*>(a.y);
      const T* pv = static_cast<const T*>(a.pv);
#pragma unroll
      for (int q = 0; q < PARTS; ++q) {
        T self[VEC], o[VEC];
        load16(x + r * NB + q * VEC, self);
#pragma unroll
        for (int j = 0; j < VEC; ++j) o[j] = al * (acc[q * VEC + j] + d * self[j]) + be * self[j];
        if (HAS_P) {
          T pq[VEC];
          load16_rw(pv + slot * NB + q * VEC, pq);
#pragma unroll
          for (int j = 0; j < VEC; ++j) o[j] += ga * pq[j];
        }
        store16(out + slot * NB + q * VEC, o);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Image tables
// ---------------------------------------------------------------------------

struct TableBuildArgs {
  SectorParams p;
  uint64_t mask;
  uint64_t dim;
  const uint64_t* states;
  const uint16_t* orbits;
  const uint8_t* class_of;  // R -> orbit class
  const uint64_t* rank_tab;
  int rank_chunks, rank_stride;
  void* table;
  int table_wide;
  int idx_bits, rbits, mbits;
  int real_phases;
};

// One thread per representative writes the entry of every image g(rep):
// column, the character of the element mapping the image back to rep, and
// the orbit class. Images reached by several elements (stabilisers) get the
// same entry, because a sector orbit's stabiliser has character 1.
__global__ void __launch_bounds__(256) image_table_build_kernel(const TableBuildArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* s_rank = reinterpret_cast<uint64_t*>(smem);
  const size_t rank_words = a.p.up >= 0 ? static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride : 0;
  for (size_t i = threadIdx.x; i < rank_words; i += blockDim.x) s_rank[i] = a.rank_tab[i];
  __syncthreads();
  const int L = a.p.sites;
  const int translations = a.p.has_momentum ? L : 1;
  const int reflections = a.p.parity != 0 ? 2 : 1;
  const int inversions = a.p.inversion != 0 ? 2 : 1;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < a.dim; i += stride) {
    const uint64_t rep = a.states[i];
    const uint64_t rclass = a.class_of[a.orbits[i]];
    for (int b = 0; b < translations; ++b) {
      const uint64_t rotated = rotate_state(rep, b, L, a.mask);
      // the image T^b rep returns to rep under T^shift
      const int shift = (L - b) % L;
      bool phase_neg = false;
      int m = 0;
      if (a.real_phases) {
        phase_neg = a.p.has_momentum && 2 * a.p.momentum == L && (shift & 1);
      } else {
        m = static_cast<int>((static_cast<long long>(a.p.momentum) * ((L - shift) % L)) % L);
      }
      for (int refl = 0; refl < reflections; ++refl) {
        for (int inv = 0; inv < inversions; ++inv) {
          uint64_t u = refl ? reflect_state(rotated, L) : rotated;
          if (inv) u = ~u & a.mask;
          const bool neg = phase_neg != ((refl && a.p.parity < 0) != (inv && a.p.inversion < 0));
          const uint64_t code = (neg ? 1ull : 0ull) | (rclass << 1) | (static_cast<uint64_t>(m) << (1 + a.rbits));
          const uint64_t entry = i | (code << a.idx_bits);
          const uint64_t rank = a.p.up >= 0 ? rank_chunked(u, s_rank, a.rank_chunks, a.rank_stride) : u;
          if (a.table_wide) static_cast<unsigned long long*>(a.table)[rank] = entry;
          else static_cast<uint32_t*>(a.table)[rank] = static_cast<uint32_t>(entry);
        }
      }
    }
  }
}

// Decodes the table entries of physical states (the images() contract:
// index or -1, character, orbit size).
__global__ void table_images_kernel(SectorParams p, const void* table, int wide, int idx_bits, int rbits, int mbits,
                                    const uint64_t* rank_tab, int chunks, int stride, const uint16_t* class_sizes,
                                    const double* phase_m, const uint64_t* lo, uint64_t n, int64_t* index,
                                    double* phase, uint16_t* orbit) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t t = lo[i];
  const uint64_t mask = low_mask<uint64_t>(p.sites);
  uint64_t e = kAllOnes;
  if ((t & ~mask) == 0 && (p.up < 0 || __popcll(t) == p.up)) {
    const uint64_t rank = p.up >= 0 ? rank_chunked(t, rank_tab, chunks, stride) : t;
    if (wide) {
      e = static_cast<const unsigned long long*>(table)[rank];
    } else {
      const uint32_t v = static_cast<const uint32_t*>(table)[rank];
      e = v == 0xffffffffu ? kAllOnes : v;
    }
  }
  if (e == kAllOnes) {
    index[i] = -1;
    phase[2 * i] = 0.0;
    phase[2 * i + 1] = 0.0;
    orbit[i] = 0;
    return;
  }
  const uint64_t code = e >> idx_bits;
  index[i] = static_cast<int64_t>(e & ((1ull << idx_bits) - 1));
  double cr = 1.0, ci = 0.0;
  if (mbits > 0) {
    const int m = static_cast<int>(code >> (1 + rbits));
    cr = phase_m[2 * m];
    ci = phase_m[2 * m + 1];
  }
  if (code & 1) {
    cr = -cr;
    ci = -ci;
  }
  phase[2 * i] = cr;
  phase[2 * i + 1] = ci;
  orbit[i] = class_sizes[(code >> 1) & ((1u << rbits) - 1)];
}

__global__ void fence_kernel(const uint64_t* states, uint64_t seg, int n, uint64_t* fences) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) fences[i] = states[static_cast<uint64_t>(i) * seg];
}

int bit_width(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

uint64_t binomial_u64(int n, int k) {
  if (k < 0 || k > n) return 0;
  k = std::min(k, n - k);
  unsigned __int128 value = 1;
  for (int i = 0; i < k; ++i) value = value * static_cast<unsigned>(n - i) / static_cast<unsigned>(i + 1);
  return value > static_cast<unsigned __int128>(UINT64_MAX) ? UINT64_MAX : static_cast<uint64_t>(value);
}

// Orbit sizes a sector can hold: period (a divisor of L, or 1 without
// translations) times 2 for a separate reflected orbit, times 2 for a
// separate spin-flipped orbit.
std::vector<int> orbit_size_classes(const SectorParams& p) {
  std::vector<int> periods;
  if (p.has_momentum) {
    for (int d = 1; d <= p.sites; ++d)
      if (p.sites % d == 0) periods.push_back(d);
  } else {
    periods.push_back(1);
  }
  std::vector<int> sizes;
  for (int per : periods)
    for (int f1 = 1; f1 <= (p.parity != 0 ? 2 : 1); ++f1)
      for (int f2 = 1; f2 <= (p.inversion != 0 ? 2 : 1); ++f2) sizes.push_back(per * f1 * f2);
  std::sort(sizes.begin(), sizes.end());
  sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
  return sizes;
}

uint64_t table_limit_bytes() {
  if (const char* env = std::getenv("QMBED_IMAGE_TABLE_MAX_BYTES")) {
    char* end = nullptr;
    const unsigned long long v = std::strtoull(env, &end, 10);
    if (end != env) return v;
  }
  return 48ull << 30;
}

}  // namespace

// ---------------------------------------------------------------------------
// SpinBasis lookup structures
// ---------------------------------------------------------------------------

void SpinBasis::prepare_lookup() {
  const SectorParams& p = params_;
  if (words() != 1) return;
  // colex chunk tables for fixed-weight spaces
  if (p.up >= 0) {
    const int chunks = (p.sites + kRankChunkBits - 1) / kRankChunkBits;
    const int stride = p.up + 1;
    const size_t words_needed = static_cast<size_t>(chunks) * kRankChunkValues * stride;
    if (words_needed * 8 <= kRankTableMaxBytes) {
      std::vector<uint64_t> tab(words_needed, 0);
      for (int c = 0; c < chunks; ++c)
        for (int v = 0; v < kRankChunkValues; ++v)
          for (int k = 0; k < stride; ++k) {
            uint64_t sum = 0;
            int ordinal = k;
            for (int b = 0; b < kRankChunkBits; ++b) {
              if (!((v >> b) & 1)) continue;
              ++ordinal;
              const int position = kRankChunkBits * c + b;
              if (position >= p.sites) break;
              sum += binomial_u64(position, ordinal);
            }
            tab[(static_cast<size_t>(c) * kRankChunkValues + v) * stride + k] = sum;
          }
      rank_tab_.allocate(tab.size() * 8);
      QMBED_CUDA(cudaMemcpy(rank_tab_.get(), tab.data(), tab.size() * 8, cudaMemcpyHostToDevice));
      rank_chunks_ = chunks;
      rank_stride_ = stride;
    }
  }
  // fence keys of the sorted representatives
  if (p.symmetric && dim_ > 0) {
    const uint64_t n = std::min<uint64_t>(kMaxFences, dim_);
    fence_seg_ = (dim_ + n - 1) / n;
    n_fences_ = static_cast<int>((dim_ + fence_seg_ - 1) / fence_seg_);
    fence_levels_ = bit_width(fence_seg_);
    fences_.allocate(static_cast<size_t>(n_fences_) * 8);
    fence_kernel<<<(n_fences_ + 255) / 256, 256>>>(states_.as<uint64_t>(), fence_seg_, n_fences_,
                                                   fences_.as<uint64_t>());
    QMBED_LAUNCH_CHECK();
  }
}

bool image_table_feasible(const SpinBasis& basis, uint64_t limit_bytes, uint64_t* bytes_out) {
  const SectorParams& p = basis.params();
  if (basis.words() != 1 || !p.symmetric || basis.dim() == 0) return false;
  if (p.up >= 0 && basis.rank_chunk_count() == 0) return false;
  if (p.up < 0 && p.sites > 36) return false;
  const uint64_t length = p.up >= 0 ? binomial_u64(p.sites, p.up) : (1ull << p.sites);
  const int idx_bits = bit_width(basis.dim());
  const int rbits = std::max(1, bit_width(orbit_size_classes(p).size() - 1));
  const int mbits = basis.real_phases() ? 0 : bit_width(static_cast<uint64_t>(p.sites - 1));
  const bool wide = idx_bits + 1 + rbits + mbits > 32;
  if (idx_bits + 1 + rbits + mbits > 64) return false;
  const uint64_t bytes = length * (wide ? 8 : 4);
  if (bytes_out) *bytes_out = bytes;
  return bytes <= limit_bytes;
}

const ImageTable* SpinBasis::image_table() const {
  std::lock_guard<std::mutex> lock(table_mu_);
  return table_.get();
}

const ImageTable* SpinBasis::build_image_table(bool required) const {
  std::lock_guard<std::mutex> lock(table_mu_);
  if (table_) return table_.get();
  uint64_t bytes = 0;
  const uint64_t limit = table_limit_bytes();
  if (!image_table_feasible(*this, limit, &bytes)) {
    if (required)
      raise(QMBED_UNSUPPORTED_BACKEND, "no image table for this sector (" + std::to_string(bytes) +
                                           " bytes; the limit is " + std::to_string(limit) + ")");
    return nullptr;
  }
  QMBED_CUDA(cudaSetDevice(device_));
  size_t free_bytes = 0, total_bytes = 0;
  QMBED_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
  if (bytes > free_bytes / 10 * 6) {
    if (required)
      raise(QMBED_UNSUPPORTED_BACKEND, "no image table for this sector: " + std::to_string(bytes) +
                                           " bytes exceed 60% of the free device memory");
    return nullptr;
  }
  auto start = std::chrono::steady_clock::now();
  auto t = std::make_unique<ImageTable>();
  const SectorParams& p = params_;
  t->length = p.up >= 0 ? binomial_u64(p.sites, p.up) : (1ull << p.sites);
  t->idx_bits = bit_width(dim_);
  const std::vector<int> classes = orbit_size_classes(p);
  t->rbits = std::max(1, bit_width(classes.size() - 1));
  t->mbits = real_phases() ? 0 : bit_width(static_cast<uint64_t>(p.sites - 1));
  t->wide = t->idx_bits + 1 + t->rbits + t->mbits > 32;
  t->bytes = t->length * (t->wide ? 8 : 4);
  t->entries.allocate(t->bytes);
  QMBED_CUDA(cudaMemset(t->entries.get(), 0xff, t->bytes));
  std::vector<uint8_t> class_of(257, 0);
  std::vector<double> class_inv_sqrt(std::max<size_t>(classes.size(), 1), 1.0);
  for (size_t c = 0; c < classes.size(); ++c) {
    if (classes[c] <= 256) class_of[static_cast<size_t>(classes[c])] = static_cast<uint8_t>(c);
    class_inv_sqrt[c] = 1.0 / std::sqrt(static_cast<double>(classes[c]));
  }
  DeviceBuffer class_of_dev(class_of.size());
  QMBED_CUDA(cudaMemcpy(class_of_dev.get(), class_of.data(), class_of.size(), cudaMemcpyHostToDevice));
  std::vector<uint16_t> class_sizes(std::max<size_t>(classes.size(), 1), 1);
  for (size_t c = 0; c < classes.size(); ++c) class_sizes[c] = static_cast<uint16_t>(classes[c]);
  t->class_sizes.allocate(class_sizes.size() * 2);
  QMBED_CUDA(cudaMemcpy(t->class_sizes.get(), class_sizes.data(), class_sizes.size() * 2, cudaMemcpyHostToDevice));
  t->class_inv_sqrt.allocate(class_inv_sqrt.size() * 8);
  QMBED_CUDA(cudaMemcpy(t->class_inv_sqrt.get(), class_inv_sqrt.data(), class_inv_sqrt.size() * 8,
                        cudaMemcpyHostToDevice));
  // m -> exp(-2 pi i m / L): the character of the shift whose reduced product k (L - shift) mod L is m
  std::vector<double> phase_m(2 * static_cast<size_t>(p.sites), 0.0);
  for (int m = 0; m < p.sites; ++m) {
    const double angle = -(2.0 * M_PI) * static_cast<double>(m) / static_cast<double>(p.sites);
    phase_m[2 * m] = m == 0 ? 1.0 : std::cos(angle);
    phase_m[2 * m + 1] = m == 0 ? 0.0 : std::sin(angle);
  }
  t->phase_m.allocate(phase_m.size() * 8);
  QMBED_CUDA(cudaMemcpy(t->phase_m.get(), phase_m.data(), phase_m.size() * 8, cudaMemcpyHostToDevice));
  TableBuildArgs a{};
  a.p = p;
  a.mask = low_mask<uint64_t>(p.sites);
  a.dim = dim_;
  a.states = states_.as<uint64_t>();
  a.orbits = orbits_.as<uint16_t>();
  a.class_of = class_of_dev.as<uint8_t>();
  a.rank_tab = rank_tab_.as<uint64_t>();
  a.rank_chunks = rank_chunks_;
  a.rank_stride = rank_stride_;
  a.table = t->entries.get();
  a.table_wide = t->wide ? 1 : 0;
  a.idx_bits = t->idx_bits;
  a.rbits = t->rbits;
  a.mbits = t->mbits;
  a.real_phases = real_phases() ? 1 : 0;
  const size_t smem = p.up >= 0 ? static_cast<size_t>(rank_chunks_) * kRankChunkValues * rank_stride_ * 8 : 0;
  int sms = 148;
  QMBED_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  const uint64_t blocks = std::min<uint64_t>((dim_ + 255) / 256, static_cast<uint64_t>(sms) * 16);
  if (smem > 48 * 1024)
    QMBED_CUDA(cudaFuncSetAttribute(image_table_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
  image_table_build_kernel<<<static_cast<unsigned>(std::max<uint64_t>(blocks, 1)), 256, smem>>>(a);
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaDeviceSynchronize());
  t->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
  table_ = std::move(t);
  return table_.get();
}

void SpinBasis::table_images(const uint64_t* lo, uint64_t n, int64_t* index, double* phase, uint16_t* orbit) const {
  QMBED_CUDA(cudaSetDevice(device_));
  const ImageTable* t = build_image_table(true);
  if (n == 0) return;
  DeviceBuffer d_lo(n * 8), d_index(n * 8), d_phase(n * 16), d_orbit(n * 2);
  QMBED_CUDA(cudaMemcpy(d_lo.get(), lo, n * 8, cudaMemcpyHostToDevice));
  table_images_kernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(
      params_, t->entries.get(), t->wide ? 1 : 0, t->idx_bits, t->rbits, t->mbits, rank_tab_.as<uint64_t>(),
      rank_chunks_, rank_stride_, t->class_sizes.as<uint16_t>(), t->phase_m.as<double>(), d_lo.as<uint64_t>(), n,
      d_index.as<int64_t>(), d_phase.as<double>(), d_orbit.as<uint16_t>());
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaMemcpy(index, d_index.get(), n * 8, cudaMemcpyDeviceToHost));
  QMBED_CUDA(cudaMemcpy(phase, d_phase.get(), n * 16, cudaMemcpyDeviceToHost));
  QMBED_CUDA(cudaMemcpy(orbit, d_orbit.get(), n * 2, cudaMemcpyDeviceToHost));
}

// ---------------------------------------------------------------------------
// Launch
// ---------------------------------------------------------------------------

namespace {

template <typename T, int NB, bool CPLX, int MODE, bool HAS_P, bool CHAIN>
void launch_chain(const TileArgs& a, size_t smem, cudaStream_t stream) {
  auto kernel = hv_tile_kernel<T, NB, CPLX, MODE, HAS_P, CHAIN>;
  // resident blocks per SM for this instantiation, cached per (device, smem)
  static thread_local int cached_device = -1;
  static thread_local size_t cached_smem = 0;
  static thread_local int cached_per_sm = 0, cached_sms = 0;
  int device = 0;
  QMBED_CUDA(cudaGetDevice(&device));
  if (cached_device != device || cached_smem != smem) {
    if (smem > 48 * 1024)
      QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    QMBED_CUDA(cudaDeviceGetAttribute(&cached_sms, cudaDevAttrMultiProcessorCount, device));
    QMBED_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_per_sm, kernel, kTileThreads, smem));
    cached_device = device;
    cached_smem = smem;
  }
  const int sms = cached_sms, per_sm = cached_per_sm;
  const uint64_t tiles = (a.rows + 31) / 32;
  const uint64_t blocks_needed = (tiles + kTileThreads / 32 - 1) / (kTileThreads / 32);
  const uint64_t cap = static_cast<uint64_t>(sms) * std::max(per_sm, 1);
  const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min(blocks_needed, cap)));
  kernel<<<grid, kTileThreads, smem, stream>>>(a);
  QMBED_LAUNCH_CHECK();
}

template <typename T, int NB, bool CPLX, int MODE, bool HAS_P>
void launch_one(const TileArgs& a, size_t smem, cudaStream_t stream, bool chain) {
  if (chain) launch_chain<T, NB, CPLX, MODE, HAS_P, true>(a, smem, stream);
  else launch_chain<T, NB, CPLX, MODE, HAS_P, false>(a, smem, stream);
}

template <typename T, int NB, bool HAS_P>
void launch_hop_kernel(const HopArgs& a, size_t smem, cudaStream_t stream) {
  auto kernel = hop_tile_kernel<T, NB, HAS_P>;
  static thread_local int cached_device = -1;
  static thread_local size_t cached_smem = 0;
  static thread_local int cached_per_sm = 0, cached_sms = 0;
  int device = 0;
  QMBED_CUDA(cudaGetDevice(&device));
  if (cached_device != device || cached_smem != smem) {
    if (smem > 48 * 1024)
      QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    QMBED_CUDA(cudaDeviceGetAttribute(&cached_sms, cudaDevAttrMultiProcessorCount, device));
    QMBED_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_per_sm, kernel, kTileThreads, smem));
    cached_device = device;
    cached_smem = smem;
  }
  const uint64_t tiles = (a.rows + 31) / 32;
  const uint64_t blocks_needed = (tiles + kTileThreads / 32 - 1) / (kTileThreads / 32);
  const uint64_t cap = static_cast<uint64_t>(cached_sms) * std::max(cached_per_sm, 1);
  const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min(blocks_needed, cap)));
  kernel<<<grid, kTileThreads, smem, stream>>>(a);
  QMBED_LAUNCH_CHECK();
}

// The hop kernel serves chain programs whose only off-diagonal class is the
// nearest-neighbour bond, on real fixed-weight sectors whose image table has
// 32-bit entries without a phase index.
bool hop_form(const SpinBasis& basis, const DeviceFlipProgram& prog, const ImageTable* table) {
  const SectorParams& p = basis.params();
  if (!table || table->wide || table->mbits != 0 || !basis.real_phases()) return false;
  if (!prog.ok() || !prog.chain_ok() || prog.complex_coefs()) return false;
  if (p.up < 0 || basis.rank_chunk_count() == 0 || p.sites < 3 || p.sites > 64) return false;
  const ChainProgram& ch = prog.chain();
  if (ch.n_off != 1 || ch.off[0].d != 1 || (ch.off[0].nz & ~0x6) != 0) return false;
  return orbit_size_classes(p).size() <= static_cast<size_t>(kHopMaxClasses);
}

bool launch_hop(const SpinBasis& basis, const DeviceFlipProgram& prog, const ImageTable& table, const TileLaunch& l) {
  const SectorParams& p = basis.params();
  const ChainProgram& ch = prog.chain();
  HopArgs a{};
  a.dim = basis.dim();
  a.row0 = l.row0;
  a.rows = std::min(l.rows, a.dim - std::min(l.row0, a.dim));
  a.sites = p.sites;
  a.up = p.up;
  a.states = static_cast<const uint64_t*>(basis.states());
  a.orbits = basis.orbits();
  a.rank_tab = basis.rank_chunk_table();
  a.rank_chunks = basis.rank_chunk_count();
  a.rank_stride = basis.rank_chunk_stride();
  a.binom = basis.binomials();
  a.table = static_cast<const uint32_t*>(table.entries.get());
  a.idx_bits = table.idx_bits;
  a.rbits = table.rbits;
  a.n_classes = static_cast<int>(orbit_size_classes(p).size());
  a.class_inv_sqrt = table.class_inv_sqrt.as<double>();
  a.inv_sqrt = l.inv_sqrt;
  const uint64_t inner = p.sites == 64 ? ~0ull >> 1 : (1ull << (p.sites - 1)) - 1;
  a.bonds_inner = ch.off[0].bonds & inner;
  a.wrap = static_cast<int>((ch.off[0].bonds >> (p.sites - 1)) & 1);
  a.w_down = ch.off[0].re[1];
  a.w_up = ch.off[0].re[2];
  a.chain = ch;
  a.x = l.x;
  a.pv = l.p;
  a.y = l.y;
  a.alpha = l.alpha;
  a.beta = l.beta;
  a.gamma = l.gamma;
  const size_t elem = l.precision == 64 ? 8 : 4;
  const size_t smem = static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride * 8 +
                      static_cast<size_t>(p.sites) * (p.up + 1) * 8 + static_cast<size_t>(a.n_classes) * elem;
  if (smem > 96 * 1024) return false;
  const bool hp = l.p != nullptr;
  if (l.nb == 1) {
    if (l.precision == 64) launch_hop_kernel<double, 1, false>(a, smem, l.stream);
    else launch_hop_kernel<float, 1, false>(a, smem, l.stream);
  } else if (l.precision == 64) {
    if (l.nb == 8) hp ? launch_hop_kernel<double, 8, true>(a, smem, l.stream)
                      : launch_hop_kernel<double, 8, false>(a, smem, l.stream);
    else hp ? launch_hop_kernel<double, 16, true>(a, smem, l.stream)
            : launch_hop_kernel<double, 16, false>(a, smem, l.stream);
  } else {
    if (l.nb == 8) hp ? launch_hop_kernel<float, 8, true>(a, smem, l.stream)
                      : launch_hop_kernel<float, 8, false>(a, smem, l.stream);
    else hp ? launch_hop_kernel<float, 16, true>(a, smem, l.stream)
            : launch_hop_kernel<float, 16, false>(a, smem, l.stream);
  }
  return true;
}

template <int MODE>
void dispatch_mode(const TileArgs& a, size_t smem, const TileLaunch& l, bool chain) {
  const bool hp = l.p != nullptr;
  if (l.nb == 1) {
    if (l.precision == 64) {
      if (l.complex_vectors) launch_one<double, 1, true, MODE, false>(a, smem, l.stream, chain);
      else launch_one<double, 1, false, MODE, false>(a, smem, l.stream, chain);
    } else {
      if (l.complex_vectors) launch_one<float, 1, true, MODE, false>(a, smem, l.stream, chain);
      else launch_one<float, 1, false, MODE, false>(a, smem, l.stream, chain);
    }
    return;
  }
  if (l.precision == 64) {
    if (l.nb == 8) hp ? launch_one<double, 8, false, MODE, true>(a, smem, l.stream, chain)
                      : launch_one<double, 8, false, MODE, false>(a, smem, l.stream, chain);
    else hp ? launch_one<double, 16, false, MODE, true>(a, smem, l.stream, chain)
            : launch_one<double, 16, false, MODE, false>(a, smem, l.stream, chain);
  } else {
    if (l.nb == 8) hp ? launch_one<float, 8, false, MODE, true>(a, smem, l.stream, chain)
                      : launch_one<float, 8, false, MODE, false>(a, smem, l.stream, chain);
    else hp ? launch_one<float, 16, false, MODE, true>(a, smem, l.stream, chain)
            : launch_one<float, 16, false, MODE, false>(a, smem, l.stream, chain);
  }
}

}  // namespace

bool hop_kernel_applies(const SpinBasis& basis, const DeviceFlipProgram& prog) {
  return hop_form(basis, prog, basis.image_table());
}

bool launch_tile(const SpinBasis& basis, const DeviceFlipProgram& prog, int mode, const TileLaunch& l) {
  if (basis.words() != 1 || !prog.ok()) return false;
  if (l.nb != 1 && l.nb != 8 && l.nb != 16) return false;
  if (l.nb != 1 && (l.complex_vectors || prog.complex_coefs() || !basis.real_phases())) return false;
  if (!l.complex_vectors && (prog.complex_coefs() || !basis.real_phases())) return false;
  const SectorParams& p = basis.params();
  TileArgs a{};
  a.p = p;
  a.mask = low_mask<uint64_t>(p.sites);
  a.dim = basis.dim();
  a.row0 = l.row0;
  a.rows = std::min(l.rows, a.dim - std::min(l.row0, a.dim));
  a.states = static_cast<const uint64_t*>(basis.states());
  a.orbits = basis.orbits();
  if (prog.bytes() > kProgramSmemMax) return false;
  a.program = static_cast<const unsigned long long*>(prog.data());
  a.program_words = static_cast<int>((prog.bytes() + 7) / 8);
  a.n_dterms = prog.n_dterms();
  a.n_terms = prog.n_terms();
  a.n_groups = prog.n_groups();
  a.n_slots = prog.n_slots();
  a.n_dpairs = prog.n_dpairs();
  a.groups_offset = static_cast<int>(prog.groups_offset());
  a.amp_offset = static_cast<int>(prog.amp_offset());
  a.pairs_offset = static_cast<int>(prog.pairs_offset());
  a.rank_tab = basis.rank_chunk_table();
  a.rank_chunks = basis.rank_chunk_count();
  a.rank_stride = basis.rank_chunk_stride();
  a.binom = basis.binomials();
  a.phase_shift = basis.phase_table();
  a.inv_sqrt = l.inv_sqrt;
  a.fences = basis.fence_keys();
  a.n_fences = basis.fence_count();
  a.fence_seg = basis.fence_segment();
  a.fence_levels = basis.fence_levels();
  a.x = l.x;
  a.pv = l.p;
  a.y = l.y;
  a.alpha = l.alpha;
  a.beta = l.beta;
  a.gamma = l.gamma;
  size_t smem = static_cast<size_t>(a.program_words) * 8;
  int tile_mode;
  if (basis.direct()) {
    tile_mode = kModeDirect;
  } else if (basis.colex()) {
    tile_mode = kModeColex;
    if (a.rank_chunks > 0) smem += static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride * 8;
  } else {
    const ImageTable* table = mode == kLookupSearch ? nullptr : basis.image_table();
    if ((mode == kLookupTable || mode == kLookupTableGeneric) && !table) return false;
    if (mode != kLookupTableGeneric && !l.complex_vectors && hop_form(basis, prog, table) &&
        launch_hop(basis, prog, *table, l))
      return true;
    if (table) {
      tile_mode = kModeTable;
      a.table = table->entries.get();
      a.table_wide = table->wide ? 1 : 0;
      a.idx_bits = table->idx_bits;
      a.rbits = table->rbits;
      a.mbits = table->mbits;
      a.class_inv_sqrt = table->class_inv_sqrt.as<double>();
      a.phase_m = table->phase_m.as<double>();
      if (p.up >= 0) smem += static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride * 8;
    } else {
      if (a.n_fences == 0) return false;
      tile_mode = kModeSearch;
      smem += static_cast<size_t>(a.n_fences) * 8;
    }
  }
  if (smem > 96 * 1024) return false;
  const bool chain = prog.chain_ok();
  if (chain) {
    a.chain = prog.chain();
    if ((tile_mode == kModeColex || tile_mode == kModeTable) && p.up >= 0 && a.rank_chunks > 0) {
      a.binom_rows = p.sites;
      smem += static_cast<size_t>(p.sites) * (p.up + 1) * 8;
      if (smem > 96 * 1024) return false;
    }
  }
  switch (tile_mode) {
    case kModeDirect: dispatch_mode<kModeDirect>(a, smem, l, chain); break;
    case kModeColex: dispatch_mode<kModeColex>(a, smem, l, chain); break;
    case kModeTable: dispatch_mode<kModeTable>(a, smem, l, chain); break;
    default: dispatch_mode<kModeSearch>(a, smem, l, chain); break;
  }
  return true;
}

}  // namespace qmbed
