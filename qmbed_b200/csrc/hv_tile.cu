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

// ---------------------------------------------------------------------------
// Flip programs (host)
// ---------------------------------------------------------------------------

FlipProgram compile_flip_program(const std::vector<Instance>& adjoint, const LocalFactors& f, int sites) {
  FlipProgram prog;
  if (sites > 64) return prog;
  // spin-1/2 factors: z(d) = z1 * (+1 | -1), ladder factors independent of d
  if (f.z[0] != -f.z[1] || f.raise != f.lower) return prog;
  std::map<uint64_t, std::map<std::tuple<uint64_t, uint64_t, uint64_t>, C64>> by_flip;
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
  for (const auto& [flip, terms] : by_flip) {
    std::vector<FlipTerm> list;
    for (const auto& [key, k] : terms) {
      if (k == C64(0.0, 0.0)) continue;
      FlipTerm t{std::get<0>(key), std::get<1>(key), std::get<2>(key), k.real(), k.imag()};
      if (t.ki != 0.0) prog.complex_coefs = true;
      list.push_back(t);
    }
    if (list.empty()) continue;
    if (flip == 0) {
      prog.diag = list;
      continue;
    }
    FlipGroup g{flip, static_cast<uint32_t>(prog.terms.size()), static_cast<uint32_t>(list.size())};
    prog.groups.push_back(g);
    prog.terms.insert(prog.terms.end(), list.begin(), list.end());
  }
  prog.ok = true;
  return prog;
}

void DeviceFlipProgram::upload(const FlipProgram& prog) {
  ok_ = prog.ok;
  if (!ok_) return;
  complex_ = prog.complex_coefs;
  n_diag_ = static_cast<int>(prog.diag.size());
  n_terms_ = n_diag_ + static_cast<int>(prog.terms.size());
  n_groups_ = static_cast<int>(prog.groups.size());
  std::vector<FlipTerm> all(prog.diag);
  all.insert(all.end(), prog.terms.begin(), prog.terms.end());
  // group term offsets are relative to the diagonal-free list: shift them
  std::vector<FlipGroup> groups(prog.groups);
  for (FlipGroup& g : groups) g.first += static_cast<uint32_t>(n_diag_);
  groups_offset_ = all.size() * sizeof(FlipTerm);
  bytes_ = groups_offset_ + groups.size() * sizeof(FlipGroup);
  buf_.allocate(std::max<size_t>(bytes_, 16));
  if (!all.empty()) QMBED_CUDA(cudaMemcpy(buf_.get(), all.data(), groups_offset_, cudaMemcpyHostToDevice));
  if (!groups.empty())
    QMBED_CUDA(cudaMemcpy(buf_.as<char>() + groups_offset_, groups.data(), groups.size() * sizeof(FlipGroup),
                          cudaMemcpyHostToDevice));
}

namespace {

constexpr int kRankChunkBits = 4;
constexpr int kRankChunkValues = 1 << kRankChunkBits;
constexpr size_t kRankTableMaxBytes = 40 * 1024;
constexpr int kMaxFences = 4096;
constexpr size_t kProgramSmemMax = 32 * 1024;
constexpr int kTileThreads = 256;
constexpr uint64_t kAllOnes = ~0ull;

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Colex rank from 4-bit chunk tables: tab[(c * 16 + v) * stride + k] is the
// rank contribution of the set bits v of chunk c when k set bits lie below
// it (fixed_weight_state_index, src/basis/mod.rs:640-659, summed per chunk).
__device__ __forceinline__ uint64_t rank_chunked(uint64_t t, const uint64_t* __restrict__ tab, int chunks,
                                                 int stride) {
  uint64_t r = 0;
  int ones = 0;
#pragma unroll 4
  for (int c = 0; c < chunks; ++c) {
    const unsigned v = static_cast<unsigned>(t >> (kRankChunkBits * c)) & (kRankChunkValues - 1);
    r += tab[(c * kRankChunkValues + v) * stride + ones];
    ones += __popc(v);
  }
  return r;
}

struct TileArgs {
  SectorParams p;
  uint64_t mask;
  uint64_t dim;
  const uint64_t* states;
  const uint16_t* orbits;
  // program
  const FlipTerm* terms;
  const FlipGroup* groups;
  int n_diag, n_terms, n_groups;
  int prog_smem;
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
};

enum TileMode : int { kModeDirect = 0, kModeColex = 1, kModeTable = 2, kModeSearch = 3 };

// Amplitude of group g (or of the diagonal when `first`..`count` span the
// diagonal terms) on state s: sum_k [s & req == val] k (-1)^popc(~s & sign).
template <bool CPLX>
__device__ __forceinline__ void group_amplitude(const FlipTerm* __restrict__ terms, uint32_t first, uint32_t count,
                                                uint64_t s, double& ar, double& ai) {
  ar = 0.0;
  ai = 0.0;
  for (uint32_t i = first; i < first + count; ++i) {
    const FlipTerm& t = terms[i];
    if ((s & t.req_mask) != t.req_val) continue;
    const bool neg = __popcll(~s & t.sign_mask) & 1;
    ar += neg ? -t.kr : t.kr;
    if (CPLX) ai += neg ? -t.ki : t.ki;
  }
}

__device__ __forceinline__ bool group_active(const FlipTerm* __restrict__ terms, uint32_t first, uint32_t count,
                                             uint64_t s) {
  bool any = false;
  for (uint32_t i = first; i < first + count; ++i) any |= (s & terms[i].req_mask) == terms[i].req_val;
  return any;
}

// Per-target lookup result: column (-1: not in the basis), character
// (chi_r, chi_i) and 1/sqrt(R_column) (1 without symmetry).
struct Hit {
  int64_t col;
  double cr, ci;
  double inv_sqrt_rc;
};

template <int U, int MODE, bool NEED_R>
__device__ __forceinline__ void lookup_batch(const TileArgs& a, const uint64_t* __restrict__ s_rank,
                                             const uint64_t* __restrict__ s_fence, const bool (&act)[U],
                                             const uint64_t (&t)[U], Hit (&h)[U]) {
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
      h[u].col = a.rank_chunks > 0 ? static_cast<int64_t>(rank_chunked(t[u], s_rank, a.rank_chunks, a.rank_stride))
                                   : colex_rank_checked(t[u], a.p.sites, a.p.up, a.binom);
    }
  } else if (MODE == kModeTable) {
    uint64_t e[U];
    // ranks first, then all table reads, so the reads are in flight together
#pragma unroll
    for (int u = 0; u < U; ++u) {
      e[u] = kAllOnes;
      if (!act[u]) continue;
      if (a.p.up >= 0 && __popcll(t[u]) != a.p.up) continue;
      const uint64_t rank = a.p.up >= 0 ? rank_chunked(t[u], s_rank, a.rank_chunks, a.rank_stride) : t[u];
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

// Gathers per target: U entries in flight per lane.
template <typename T, int NB, bool CPLX>
struct TileShape {
  static constexpr int U = NB == 1 ? 8 : (NB * sizeof(T) <= 32 ? 4 : (NB * sizeof(T) <= 64 ? 2 : 1));
};

// One warp per tile of 32 consecutive rows, one lane per row. Each lane
// marks its row's active flip groups in a bit mask; the warp then pops U
// groups per lane per round, so every lane stays busy until the row with the
// most transitions in the tile is done. NB = 1 computes y = H x (orbit ratio
// sqrt(R_r / R_c) applied, x real or interleaved complex); NB = 8/16 computes
// the block action in orbit-scaled coordinates with the three-term epilogue.
template <typename T, int NB, bool CPLX, int MODE, bool HAS_P>
__global__ void __launch_bounds__(kTileThreads, 2) hv_tile_kernel(const TileArgs a) {
  constexpr int U = TileShape<T, NB, CPLX>::U;
  constexpr bool NEED_R = NB == 1;
  constexpr int VEC = 16 / sizeof(T);
  constexpr int PARTS = NB >= VEC ? NB / VEC : 1;
  extern __shared__ __align__(16) unsigned char smem[];
  // shared memory: [program terms][groups][rank chunk table][fence keys]
  const size_t prog_bytes = a.prog_smem ? a.n_terms * sizeof(FlipTerm) + a.n_groups * sizeof(FlipGroup) : 0;
  const size_t rank_words = (MODE == kModeColex || MODE == kModeTable) && a.rank_chunks > 0
                                ? static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride
                                : 0;
  unsigned long long* words = reinterpret_cast<unsigned long long*>(smem);
  if (a.prog_smem) {
    const unsigned long long* src_t = reinterpret_cast<const unsigned long long*>(a.terms);
    const size_t tw = a.n_terms * sizeof(FlipTerm) / 8;
    for (size_t i = threadIdx.x; i < tw; i += blockDim.x) words[i] = src_t[i];
    const unsigned long long* src_g = reinterpret_cast<const unsigned long long*>(a.groups);
    const size_t gw = a.n_groups * sizeof(FlipGroup) / 8;
    for (size_t i = threadIdx.x; i < gw; i += blockDim.x) words[tw + i] = src_g[i];
  }
  uint64_t* s_rank = reinterpret_cast<uint64_t*>(smem + prog_bytes);
  for (size_t i = threadIdx.x; i < rank_words; i += blockDim.x) s_rank[i] = a.rank_tab[i];
  uint64_t* s_fence = s_rank + rank_words;
  if (MODE == kModeSearch)
    for (int i = threadIdx.x; i < a.n_fences; i += blockDim.x) s_fence[i] = a.fences[i];
  __syncthreads();
  const FlipTerm* terms = a.prog_smem ? reinterpret_cast<const FlipTerm*>(smem) : a.terms;
  const FlipGroup* groups =
      a.prog_smem ? reinterpret_cast<const FlipGroup*>(smem + a.n_terms * sizeof(FlipTerm)) : a.groups;

  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const T* x = static_cast<const T*>(a.x);
  for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 32 < a.dim;
       tile += warps) {
    const uint64_t r = tile * 32 + lane;
    const bool valid = r < a.dim;
    uint64_t s = 0;
    if (valid) s = MODE == kModeDirect ? r : __ldcs(a.states + r);
    double dr = 0.0, di = 0.0;
    if (valid) group_amplitude<CPLX>(terms, 0, a.n_diag, s, dr, di);
    T acc[NB], acc_i = 0;
#pragma unroll
    for (int j = 0; j < NB; ++j) acc[j] = 0;
    for (int g0 = 0; g0 < a.n_groups; g0 += 64) {
      const int gn = min(64, a.n_groups - g0);
      uint64_t active = 0;
      if (valid)
        for (int g = 0; g < gn; ++g) {
          const FlipGroup grp = groups[g0 + g];
          if (group_active(terms, grp.first, grp.count, s)) active |= 1ull << g;
        }
      while (__any_sync(0xffffffffu, active != 0)) {
        bool act[U];
        uint64_t t[U];
        double wr[U], wi[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          act[u] = active != 0;
          t[u] = 0;
          wr[u] = 0.0;
          wi[u] = 0.0;
          if (!act[u]) continue;
          const int g = __ffsll(static_cast<long long>(active)) - 1;
          active &= active - 1;
          const FlipGroup grp = groups[g0 + g];
          group_amplitude<CPLX>(terms, grp.first, grp.count, s, wr[u], wi[u]);
          t[u] = s ^ grp.flip;
        }
        Hit h[U];
        lookup_batch<U, MODE, NEED_R>(a, s_rank, s_fence, act, t, h);
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
            // w * chi / sqrt(R_c)
            const double fr = (wr[u] * h[u].cr - wi[u] * h[u].ci) * h[u].inv_sqrt_rc;
            const double fi = (wr[u] * h[u].ci + wi[u] * h[u].cr) * h[u].inv_sqrt_rc;
            if (CPLX) {
              acc[0] += static_cast<T>(fr) * gr[u] - static_cast<T>(fi) * gi[u];
              acc_i += static_cast<T>(fr) * gi[u] + static_cast<T>(fi) * gr[u];
            } else {
              acc[0] += static_cast<T>(fr) * gr[u];
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
    }
    if (!valid) continue;
    if (NB == 1) {
      const T scale = a.p.symmetric ? static_cast<T>(__ldg(a.inv_sqrt + 257 + __ldcs(a.orbits + r))) : static_cast<T>(1);
      T* y = static_cast<T*>(a.y);
      if (CPLX) {
        const T xr = __ldcs(x + 2 * r), xi = __ldcs(x + 2 * r + 1);
        const T d_r = static_cast<T>(dr), d_i = static_cast<T>(di);
        __stcs(y + 2 * r, scale * acc[0] + d_r * xr - d_i * xi);
        __stcs(y + 2 * r + 1, scale * acc_i + d_r * xi + d_i * xr);
      } else {
        __stcs(y + r, scale * acc[0] + static_cast<T>(dr) * __ldcs(x + r));
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
          load16_rw(pv + r * NB + q * VEC, pq);
#pragma unroll
          for (int j = 0; j < VEC; ++j) o[j] += ga * pq[j];
        }
        store16(out + r * NB + q * VEC, o);
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

template <typename T, int NB, bool CPLX, int MODE, bool HAS_P>
void launch_one(const TileArgs& a, size_t smem, cudaStream_t stream) {
  auto kernel = hv_tile_kernel<T, NB, CPLX, MODE, HAS_P>;
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
  const uint64_t tiles = (a.dim + 31) / 32;
  const uint64_t blocks_needed = (tiles + kTileThreads / 32 - 1) / (kTileThreads / 32);
  const uint64_t cap = static_cast<uint64_t>(sms) * std::max(per_sm, 1);
  const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min(blocks_needed, cap)));
  kernel<<<grid, kTileThreads, smem, stream>>>(a);
  QMBED_LAUNCH_CHECK();
}

template <int MODE>
void dispatch_mode(const TileArgs& a, size_t smem, const TileLaunch& l) {
  const bool hp = l.p != nullptr;
  if (l.nb == 1) {
    if (l.precision == 64) {
      if (l.complex_vectors) launch_one<double, 1, true, MODE, false>(a, smem, l.stream);
      else launch_one<double, 1, false, MODE, false>(a, smem, l.stream);
    } else {
      if (l.complex_vectors) launch_one<float, 1, true, MODE, false>(a, smem, l.stream);
      else launch_one<float, 1, false, MODE, false>(a, smem, l.stream);
    }
    return;
  }
  if (l.precision == 64) {
    if (l.nb == 8) hp ? launch_one<double, 8, false, MODE, true>(a, smem, l.stream)
                      : launch_one<double, 8, false, MODE, false>(a, smem, l.stream);
    else hp ? launch_one<double, 16, false, MODE, true>(a, smem, l.stream)
            : launch_one<double, 16, false, MODE, false>(a, smem, l.stream);
  } else {
    if (l.nb == 8) hp ? launch_one<float, 8, false, MODE, true>(a, smem, l.stream)
                      : launch_one<float, 8, false, MODE, false>(a, smem, l.stream);
    else hp ? launch_one<float, 16, false, MODE, true>(a, smem, l.stream)
            : launch_one<float, 16, false, MODE, false>(a, smem, l.stream);
  }
}

}  // namespace

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
  a.states = static_cast<const uint64_t*>(basis.states());
  a.orbits = basis.orbits();
  a.terms = prog.terms();
  a.groups = prog.groups();
  a.n_diag = prog.n_diag();
  a.n_terms = prog.n_terms();
  a.n_groups = prog.n_groups();
  a.prog_smem = prog.bytes() <= kProgramSmemMax ? 1 : 0;
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
  size_t smem = a.prog_smem ? prog.bytes() : 0;
  int tile_mode;
  if (basis.direct()) {
    tile_mode = kModeDirect;
  } else if (basis.colex()) {
    tile_mode = kModeColex;
    if (a.rank_chunks > 0) smem += static_cast<size_t>(a.rank_chunks) * kRankChunkValues * a.rank_stride * 8;
  } else {
    const ImageTable* table = mode == kLookupSearch ? nullptr : basis.image_table();
    if (mode == kLookupTable && !table) return false;
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
  switch (tile_mode) {
    case kModeDirect: dispatch_mode<kModeDirect>(a, smem, l); break;
    case kModeColex: dispatch_mode<kModeColex>(a, smem, l); break;
    case kModeTable: dispatch_mode<kModeTable>(a, smem, l); break;
    default: dispatch_mode<kModeSearch>(a, smem, l); break;
  }
  return true;
}

}  // namespace qmbed
