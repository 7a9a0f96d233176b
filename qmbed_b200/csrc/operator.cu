// Term expansion, matrix-free H.v (kernel K4), packed-CSR assembly and SpMV.
//
// Reference behaviour (matrixlab-research/QMBED):
//   visit_unreduced_local_transitions_with_symbols  src/basis/mod.rs:1122-1232
//   index_transition (sqrt(R_src/R_tgt) conj(phase))  src/basis/mod.rs:1561-1580
//   OperatorBuilder::build (column streaming, coalesce, drop |v|<=eps) src/operator/mod.rs:2091-2216
//   is_hermitian(1e-12)                               src/operator/mod.rs:1313-1398
//   apply / apply_real                                src/operator/mod.rs:1401-1548
//
// The reference builds column c of H by expanding the terms on the state of
// c. Here row r of H is built by expanding the adjoint terms on the state of
// r and conjugating: H[r,c] = conj(H^dag[c,r]). This is exact for any
// operator and gives a gather (one writer per output row, no atomics).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "device_util.cuh"
#include "krylov.cuh"
#include "operator.cuh"

namespace qmbed {

namespace {

constexpr int kRowCap = 128;               // off-diagonal transitions per row held while assembling
constexpr int kDictSlots = 4096;           // value dictionary (open addressing)
constexpr int kMaxCodes = 1024;
constexpr unsigned long long kDictEmpty = 0xFFFFFFFFFFFFFFFFULL;
constexpr int kSmemInstances = 1024;

enum DeviceFlag : int { kFlagRowOverflow = 1, kFlagDictOverflow = 2, kFlagNonHermitian = 4 };

template <typename S>
struct OpView {
  SectorParams p;
  S mask;
  const S* states;
  const uint16_t* orbits;
  uint64_t dim;
  int direct, colex;
  const uint64_t* binom;
  const double* phase;     // 2L: exp(2 pi i k a / L)
  const double* inv_sqrt;  // [R] -> 1/sqrt(R), R <= 256; [257 + R] -> sqrt(R)
  const Instance* inst;
  int n_inst;
  LocalFactors f;
};

template <typename S>
__host__ __device__ inline S row_state(const OpView<S>& v, uint64_t r) {
  return v.direct ? static_cast<S>(r) : v.states[r];
}

// Applies one product to `s` right to left; false when the action is zero.
template <typename S>
__host__ __device__ inline bool apply_instance(const Instance& in, S s, const LocalFactors& f, S& t, double& ar, double& ai) {
  t = s;
  ar = 1.0;
  ai = 0.0;
  for (int q = in.n - 1; q >= 0; --q) {
    const int site = in.site[q];
    const S bit = static_cast<S>(1) << site;
    const int d = static_cast<int>((t >> site) & 1);
    switch (in.sym[q]) {
      case 'z': {
        const double z = f.z[d];
        ar *= z;
        ai *= z;
        break;
      }
      case '+':
        if (d) return false;
        t |= bit;
        ar *= f.raise;
        ai *= f.raise;
        break;
      case '-':
        if (!d) return false;
        t &= ~bit;
        ar *= f.lower;
        ai *= f.lower;
        break;
      case 'x': {
        const double g = f.xy_scale * (d ? f.lower : f.raise);
        t ^= bit;
        ar *= g;
        ai *= g;
        break;
      }
      case 'y': {
        const double g = f.xy_scale * (d ? f.lower : f.raise);
        t ^= bit;
        const double nr = d ? -ai * g : ai * g;
        const double ni = d ? ar * g : -ar * g;
        ar = nr;
        ai = ni;
        break;
      }
      default:
        break;  // identity
    }
  }
  return true;
}

struct Located {
  int64_t col;
  double pr, pi;
  int orbit;
};

template <typename S>
__host__ __device__ inline Located locate(const OpView<S>& v, S t) {
  Located out{-1, 1.0, 0.0, 1};
  if ((t & ~v.mask) != 0) return out;
  if (v.direct) {
    out.col = static_cast<uint64_t>(t) < v.dim ? static_cast<int64_t>(t) : -1;
    return out;
  }
  if (v.colex) {
    out.col = colex_rank_checked(t, v.p.sites, v.p.up, v.binom);
    return out;
  }
  Canonical<S> c = canonicalize(t, v.p, v.mask);
  out.col = find_sorted(v.states, v.dim, c.rep);
  if (out.col >= 0) {
    out.pr = v.phase[2 * c.shift];
    out.pi = v.phase[2 * c.shift + 1];
    if ((c.reflected && v.p.parity < 0) != (c.inverted && v.p.inversion < 0)) {
      out.pr = -out.pr;
      out.pi = -out.pi;
    }
    out.orbit = v.orbits[out.col];
  }
  return out;
}

template <typename T>
struct VecIO;
template <>
struct VecIO<double> {
  using Acc = double;
};
template <>
struct VecIO<float> {
  using Acc = float;
};

// Matrix-free y = H x: one thread per row, adjoint terms expanded on the fly.
template <typename S, typename T, bool CPLX>
__global__ void __launch_bounds__(256) hv_matrix_free_kernel(OpView<S> v, const T* __restrict__ x,
                                                             T* __restrict__ y) {
  extern __shared__ Instance shared_inst[];
  const bool in_smem = v.n_inst <= kSmemInstances;
  if (in_smem)
    for (int k = threadIdx.x; k < v.n_inst; k += blockDim.x) shared_inst[k] = v.inst[k];
  __syncthreads();
  const Instance* inst = in_smem ? shared_inst : v.inst;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    const S s = row_state(v, r);
    const double sqrt_r = v.p.symmetric ? v.inv_sqrt[257 + v.orbits[r]] : 1.0;
    T acc_r = 0, acc_i = 0;
    T xr_r, xr_i = 0;
    if (CPLX) {
      xr_r = x[2 * r];
      xr_i = x[2 * r + 1];
    } else {
      xr_r = x[r];
    }
    for (int k = 0; k < v.n_inst; ++k) {
      S t;
      double ar, ai;
      if (!apply_instance(inst[k], s, v.f, t, ar, ai)) continue;
      // conj(coefficient * amplitude)
      const double wr = inst[k].cr * ar - inst[k].ci * ai;
      const double wi = -(inst[k].cr * ai + inst[k].ci * ar);
      if (t == s) {
        if (CPLX) {
          acc_r += static_cast<T>(wr) * xr_r - static_cast<T>(wi) * xr_i;
          acc_i += static_cast<T>(wr) * xr_i + static_cast<T>(wi) * xr_r;
        } else {
          acc_r += static_cast<T>(wr) * xr_r;
        }
        continue;
      }
      const Located L = locate(v, t);
      if (L.col < 0) continue;
      const double ratio = v.p.symmetric ? sqrt_r * v.inv_sqrt[L.orbit] : 1.0;
      const double fr = (wr * L.pr - wi * L.pi) * ratio;
      const double fi = (wr * L.pi + wi * L.pr) * ratio;
      if (CPLX) {
        const T xc_r = x[2 * L.col], xc_i = x[2 * L.col + 1];
        acc_r += static_cast<T>(fr) * xc_r - static_cast<T>(fi) * xc_i;
        acc_i += static_cast<T>(fr) * xc_i + static_cast<T>(fi) * xc_r;
      } else {
        acc_r += static_cast<T>(fr) * x[L.col];
      }
    }
    if (CPLX) {
      y[2 * r] = acc_r;
      y[2 * r + 1] = acc_i;
    } else {
      y[r] = acc_r;
    }
  }
}

// Per-row transition list in H-row form: entries (c, conj(coef*amp)*phase[*ratio]).
struct RowList {
  uint32_t col[kRowCap];
  double re[kRowCap];
  double im[kRowCap];
  int count;
  double diag_re, diag_im;
  int overflow;
};

// Stable insertion sort by column, then equal columns added in the order they
// were collected (so a row's sums do not depend on when this runs).
__host__ __device__ inline void sort_coalesce(RowList& out) {
  for (int i = 1; i < out.count; ++i) {
    const uint32_t c = out.col[i];
    const double a = out.re[i], b = out.im[i];
    int j = i - 1;
    while (j >= 0 && out.col[j] > c) {
      out.col[j + 1] = out.col[j];
      out.re[j + 1] = out.re[j];
      out.im[j + 1] = out.im[j];
      --j;
    }
    out.col[j + 1] = c;
    out.re[j + 1] = a;
    out.im[j + 1] = b;
  }
  int m = 0;
  for (int i = 0; i < out.count; ++i) {
    if (m > 0 && out.col[m - 1] == out.col[i]) {
      out.re[m - 1] += out.re[i];
      out.im[m - 1] += out.im[i];
    } else {
      out.col[m] = out.col[i];
      out.re[m] = out.re[i];
      out.im[m] = out.im[i];
      ++m;
    }
  }
  out.count = m;
}

// Expands `inst` on row r. With `with_ratio`, entries carry sqrt(R_r/R_c) and
// the diagonal is kept as an ordinary entry; otherwise the ratio is left out
// (the packed format applies it through the scaled input vector) and the
// diagonal is returned separately. Entries are sorted by column and coalesced.
template <typename S>
__host__ __device__ inline void collect_row(const OpView<S>& v, const Instance* inst, int n_inst, uint64_t r, bool with_ratio,
                                   RowList& out) {
  const S s = row_state(v, r);
  const double sqrt_r = v.p.symmetric ? v.inv_sqrt[257 + v.orbits[r]] : 1.0;
  out.count = 0;
  out.diag_re = 0.0;
  out.diag_im = 0.0;
  out.overflow = 0;
  for (int k = 0; k < n_inst; ++k) {
    S t;
    double ar, ai;
    if (!apply_instance(inst[k], s, v.f, t, ar, ai)) continue;
    const double wr = inst[k].cr * ar - inst[k].ci * ai;
    const double wi = -(inst[k].cr * ai + inst[k].ci * ar);
    if (t == s) {
      out.diag_re += wr;
      out.diag_im += wi;
      continue;
    }
    const Located L = locate(v, t);
    if (L.col < 0) continue;
    double fr = wr * L.pr - wi * L.pi;
    double fi = wr * L.pi + wi * L.pr;
    if (static_cast<uint64_t>(L.col) == r) {
      out.diag_re += fr;
      out.diag_im += fi;
      continue;
    }
    if (with_ratio) {
      const double ratio = v.p.symmetric ? sqrt_r * v.inv_sqrt[L.orbit] : 1.0;
      fr *= ratio;
      fi *= ratio;
    }
    if (out.count == kRowCap) {
      sort_coalesce(out);  // the buffer holds kRowCap distinct columns at most
      if (out.count == kRowCap) {
        out.overflow = 1;
        continue;
      }
    }
    out.col[out.count] = static_cast<uint32_t>(L.col);
    out.re[out.count] = fr;
    out.im[out.count] = fi;
    ++out.count;
  }
  sort_coalesce(out);
}

// |H[r,c]| <= eps entries are not stored (reference drop rule, mod.rs:2162-2164).
template <typename S>
__host__ __device__ inline bool keep_entry(const OpView<S>& v, uint64_t r, const RowList& row, int i) {
  double ratio = 1.0;
  if (v.p.symmetric) ratio = v.inv_sqrt[257 + v.orbits[r]] * v.inv_sqrt[v.orbits[row.col[i]]];
  return hypot(row.re[i], row.im[i]) * ratio > 2.220446049250313e-16;
}

__device__ inline unsigned long long value_key(double value) {
  return value == 0.0 ? 0ULL : static_cast<unsigned long long>(__double_as_longlong(value));
}

__device__ inline unsigned dict_hash(unsigned long long key) {
  key ^= key >> 33;
  key *= 0xff51afd7ed558ccdULL;
  key ^= key >> 33;
  return static_cast<unsigned>(key);
}

__device__ inline void dict_insert(unsigned long long* keys, double value, int* flags) {
  const unsigned long long key = value_key(value);
  unsigned h = dict_hash(key) & (kDictSlots - 1);
  for (int probe = 0; probe < kDictSlots; ++probe) {
    const unsigned long long prev = atomicCAS(keys + h, kDictEmpty, key);
    if (prev == kDictEmpty || prev == key) return;
    h = (h + 1) & (kDictSlots - 1);
  }
  atomicOr(flags, kFlagDictOverflow);
}

__device__ inline int dict_code(const unsigned long long* keys, const int16_t* codes, double value) {
  const unsigned long long key = value_key(value);
  unsigned h = dict_hash(key) & (kDictSlots - 1);
  for (int probe = 0; probe < kDictSlots; ++probe) {
    if (keys[h] == key) return codes[h];
    if (keys[h] == kDictEmpty) return -1;
    h = (h + 1) & (kDictSlots - 1);
  }
  return -1;
}

template <typename S>
__global__ void __launch_bounds__(128) assemble_count_kernel(OpView<S> v, uint32_t* row_nnz, double* diag,
                                                             unsigned long long* dict, int use_dict, int* flags) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  RowList row;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    collect_row(v, v.inst, v.n_inst, r, false, row);
    if (row.overflow) atomicOr(flags, kFlagRowOverflow);
    uint32_t kept = 0;
    for (int i = 0; i < row.count; ++i) {
      if (!keep_entry(v, r, row, i)) continue;
      ++kept;
      if (use_dict) dict_insert(dict, row.re[i], flags);
    }
    row_nnz[r] = kept;
    const bool keep_diag = hypot(row.diag_re, row.diag_im) > 2.220446049250313e-16;
    diag[2 * r] = keep_diag ? row.diag_re : 0.0;
    diag[2 * r + 1] = keep_diag ? row.diag_im : 0.0;
  }
}

template <typename S, typename IDX>
__global__ void __launch_bounds__(128) assemble_fill_kernel(OpView<S> v, const IDX* row_ptr, uint32_t* entries,
                                                            double* values, const unsigned long long* dict,
                                                            const int16_t* codes, int col_bits, int* flags) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  RowList row;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    collect_row(v, v.inst, v.n_inst, r, false, row);
    IDX out = row_ptr[r];
    for (int i = 0; i < row.count; ++i) {
      if (!keep_entry(v, r, row, i)) continue;
      if (codes) {
        const int code = dict_code(dict, codes, row.re[i]);
        if (code < 0) atomicOr(flags, kFlagDictOverflow);
        entries[out] = row.col[i] | (static_cast<uint32_t>(code < 0 ? 0 : code) << col_bits);
      } else {
        entries[out] = row.col[i];
        values[2 * static_cast<uint64_t>(out)] = row.re[i];
        values[2 * static_cast<uint64_t>(out) + 1] = row.im[i];
      }
      ++out;
    }
  }
}

// Row r of H (from the adjoint terms) must equal row r of H^dag (from the
// forward terms) entry by entry within 1e-12.
template <typename S>
__global__ void __launch_bounds__(128) hermitian_check_kernel(OpView<S> v, const Instance* fwd, int* flags) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  RowList a, b;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    collect_row(v, v.inst, v.n_inst, r, true, a);
    collect_row(v, fwd, v.n_inst, r, true, b);
    if (a.overflow || b.overflow) atomicOr(flags, kFlagRowOverflow);
    bool ok = hypot(a.diag_re - b.diag_re, a.diag_im - b.diag_im) <= 1.0e-12;
    int i = 0, j = 0;
    while (ok && (i < a.count || j < b.count)) {
      double dr, di;
      if (j >= b.count || (i < a.count && a.col[i] < b.col[j])) {
        dr = a.re[i];
        di = a.im[i];
        ++i;
      } else if (i >= a.count || b.col[j] < a.col[i]) {
        dr = b.re[j];
        di = b.im[j];
        ++j;
      } else {
        dr = a.re[i] - b.re[j];
        di = a.im[i] - b.im[j];
        ++i;
        ++j;
      }
      ok = hypot(dr, di) <= 1.0e-12;
    }
    if (!ok) atomicOr(flags, kFlagNonHermitian);
  }
}

// Column sums of |H| off the diagonal and the diagonal itself, per column c,
// from the forward terms (row c of H^dag holds conj(H[., c])).
template <typename S>
__global__ void __launch_bounds__(128) column_norm_kernel(OpView<S> v, const Instance* fwd, double* diag,
                                                          double* offsum, int* flags) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  RowList row;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    collect_row(v, fwd, v.n_inst, r, true, row);
    if (row.overflow) atomicOr(flags, kFlagRowOverflow);
    double sum = 0.0;
    for (int i = 0; i < row.count; ++i) {
      const double m = hypot(row.re[i], row.im[i]);
      if (m > 2.220446049250313e-16) sum += m;
    }
    offsum[r] = sum;
    // diagonal of H is conj of the H^dag diagonal
    diag[2 * r] = row.diag_re;
    diag[2 * r + 1] = -row.diag_im;
  }
}

template <typename T>
struct Pair;
template <>
struct Pair<float> {
  using type = float2;
};
template <>
struct Pair<double> {
  using type = double2;
};

// y[r] = sqrt(R_r) * sum_k table[code_k] * xs[col_k] + d[r] * x[r]  (real operators).
// With CPLX the vectors are interleaved complex and each gather reads the
// (re, im) pair of a column as one 8/16-byte load.
template <typename T, typename IDX, bool SCALED, int LANES, bool CPLX>
__global__ void __launch_bounds__(256) spmv_packed_kernel(uint64_t n, const IDX* __restrict__ row_ptr,
                                                          const uint32_t* __restrict__ entries, int col_bits,
                                                          const double* __restrict__ code_values, int n_codes,
                                                          const T* __restrict__ diag,
                                                          const uint16_t* __restrict__ orbits,
                                                          const double* __restrict__ sqrt_table,
                                                          const T* __restrict__ xs, const T* __restrict__ x,
                                                          T* __restrict__ y) {
  using P2 = typename Pair<T>::type;
  __shared__ T table[kMaxCodes];
  __shared__ T sqrt_r[257];
  for (int i = threadIdx.x; i < n_codes; i += blockDim.x) table[i] = static_cast<T>(code_values[i]);
  if (SCALED)
    for (int i = threadIdx.x; i < 257; i += blockDim.x) sqrt_r[i] = static_cast<T>(sqrt_table[257 + i]);
  __syncthreads();
  const uint32_t col_mask = col_bits >= 32 ? 0xffffffffu : ((1u << col_bits) - 1u);
  const int lane = threadIdx.x % LANES;
  // the lanes of one row shuffle among themselves only
  const unsigned group_mask = (LANES == 32 ? 0xffffffffu : ((1u << LANES) - 1u)) << ((threadIdx.x & 31) / LANES * LANES);
  const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LANES;
  const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / LANES;
  constexpr int kBatch = 4;  // entries per lane issued together: loads, then gathers, then FMAs
  for (uint64_t r = group; r < n; r += groups) {
    // Streamed arrays (row pointers, entries, diagonal, x, orbits) are read
    // evict-first so the L2 keeps the gathered vector xs.
    const IDX begin = __ldcs(row_ptr + r), end = __ldcs(row_ptr + r + 1);
    // per-row operands requested before the entry loop so their latency overlaps it
    T d = 0, xr = 0, xi = 0;
    uint16_t orbit = 0;
    if (lane == 0) {
      d = __ldcs(diag + r);
      if (CPLX) {
        const P2 v = __ldcs(reinterpret_cast<const P2*>(x) + r);
        xr = v.x;
        xi = v.y;
      } else {
        xr = __ldcs(x + r);
      }
      if (SCALED) orbit = __ldcs(orbits + r);
    }
    T acc = 0, acc_i = 0;
    for (IDX p0 = begin + lane; p0 < end; p0 += LANES * kBatch) {
      uint32_t e[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const IDX p = p0 + u * LANES;
        e[u] = p < end ? __ldcs(entries + p) : 0u;
      }
      if (CPLX) {
        P2 g[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          if (p0 + u * LANES < end) {
            g[u] = reinterpret_cast<const P2*>(xs)[e[u] & col_mask];
          } else {
            g[u].x = 0;
            g[u].y = 0;
          }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
          if (p0 + u * LANES < end) {
            const T c = table[e[u] >> col_bits];
            acc += c * g[u].x;
            acc_i += c * g[u].y;
          }
      } else {
        T g[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) g[u] = (p0 + u * LANES < end) ? xs[e[u] & col_mask] : static_cast<T>(0);
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
          if (p0 + u * LANES < end) acc += table[e[u] >> col_bits] * g[u];
      }
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(group_mask, acc, o, LANES);
      if (CPLX) acc_i += __shfl_xor_sync(group_mask, acc_i, o, LANES);
    }
    if (lane == 0) {
      const T scale = SCALED ? sqrt_r[orbit] : static_cast<T>(1);
      if (CPLX) {
        P2 out;
        out.x = scale * acc + d * xr;
        out.y = scale * acc_i + d * xi;
        __stcs(reinterpret_cast<P2*>(y) + r, out);
      } else {
        __stcs(y + r, scale * acc + d * xr);
      }
    }
  }
}

// Explicit-value rows (complex or many-valued operators): interleaved complex.
template <typename T, typename IDX, bool SCALED, int LANES, bool CPLX>
__global__ void __launch_bounds__(256) spmv_wide_kernel(uint64_t n, const IDX* __restrict__ row_ptr,
                                                        const uint32_t* __restrict__ cols,
                                                        const T* __restrict__ values, const T* __restrict__ diag,
                                                        const uint16_t* __restrict__ orbits,
                                                        const double* __restrict__ sqrt_table,
                                                        const T* __restrict__ xs, const T* __restrict__ x,
                                                        T* __restrict__ y) {
  const int lane = threadIdx.x % LANES;
  const unsigned group_mask = (LANES == 32 ? 0xffffffffu : ((1u << LANES) - 1u)) << ((threadIdx.x & 31) / LANES * LANES);
  const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LANES;
  const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / LANES;
  for (uint64_t r = group; r < n; r += groups) {
    T ar = 0, ai = 0;
    const IDX begin = row_ptr[r], end = row_ptr[r + 1];
    for (IDX p = begin + lane; p < end; p += LANES) {
      const uint32_t c = __ldg(cols + p);
      const T vr = values[2 * static_cast<uint64_t>(p)];
      if (CPLX) {
        const T vi = values[2 * static_cast<uint64_t>(p) + 1];
        const T xr = xs[2 * static_cast<uint64_t>(c)], xi = xs[2 * static_cast<uint64_t>(c) + 1];
        ar += vr * xr - vi * xi;
        ai += vr * xi + vi * xr;
      } else {
        ar += vr * xs[c];
      }
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) {
      ar += __shfl_xor_sync(group_mask, ar, o, LANES);
      ai += __shfl_xor_sync(group_mask, ai, o, LANES);
    }
    if (lane == 0) {
      const T scale = SCALED ? static_cast<T>(sqrt_table[257 + orbits[r]]) : static_cast<T>(1);
      if (CPLX) {
        const T dr = diag[2 * r], di = diag[2 * r + 1];
        const T xr = x[2 * r], xi = x[2 * r + 1];
        y[2 * r] = scale * ar + dr * xr - di * xi;
        y[2 * r + 1] = scale * ai + dr * xi + di * xr;
      } else {
        y[r] = scale * ar + diag[r] * x[r];
      }
    }
  }
}

// Block action in orbit-scaled coordinates on row-major blocks of NB columns.
// With z = x / sqrt(R) the stored rows give (S^-1 H S z)_r = sum_k c_k z_col + d_r z_r,
// so no orbit factor appears in the loop. Per row:
//   out[r][:] = alpha * (sum_k table[code_k] z[col_k][:] + d_r z[r][:]) + beta * z[r][:] + gamma * p[r][:]
// which is one step of a three-term (Chebyshev) recurrence. A row's NB values
// are LPR consecutive 16-byte vectors, one per lane, so the gather of a column
// is one contiguous NB-element read shared by LPR lanes. ES lane groups split
// the row's entries between them (partial sums combined by shuffles within
// the row's lanes) and each lane issues KB entry loads, then KB gathers, before
// its FMAs: both raise the loads in flight per warp. `out` may alias `p`
// (each row is read before it is written by the same lane), never `z`.
template <typename T, typename IDX, int NB, bool HAS_P, int ES, int KB>
__global__ void __launch_bounds__(256) spmm_packed_kernel(uint64_t n, const IDX* __restrict__ row_ptr,
                                                          const uint32_t* __restrict__ entries, int col_bits,
                                                          const double* __restrict__ code_values, int n_codes,
                                                          const T* __restrict__ diag, const T* __restrict__ z,
                                                          const T* p, T* out, T alpha, T beta, T gamma) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr int LPR = NB / VEC;
  constexpr int G = LPR * ES;  // lanes per row
  static_assert(NB % VEC == 0 && G <= 32 && 32 % G == 0, "a row's lanes must tile a warp");
  __shared__ T table[kMaxCodes];
  for (int i = threadIdx.x; i < n_codes; i += blockDim.x) table[i] = static_cast<T>(code_values[i]);
  __syncthreads();
  const uint32_t col_mask = col_bits >= 32 ? 0xffffffffu : ((1u << col_bits) - 1u);
  const int gl = threadIdx.x % G;
  const int part = gl % LPR, split = gl / LPR;
  const unsigned group_mask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << ((threadIdx.x & 31) / G * G);
  const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
  const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / G;
  for (uint64_t r = group; r < n; r += groups) {
    const IDX begin = __ldcs(row_ptr + r), end = __ldcs(row_ptr + r + 1);
    T acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = 0;
    for (IDX p0 = begin + split; p0 < end; p0 += ES * KB) {
      uint32_t e[KB];
#pragma unroll
      for (int u = 0; u < KB; ++u) e[u] = p0 + u * ES < end ? __ldcs(entries + p0 + u * ES) : 0u;
      T g[KB][VEC];
#pragma unroll
      for (int u = 0; u < KB; ++u) {
        if (p0 + u * ES < end) {
          load16(z + static_cast<uint64_t>(e[u] & col_mask) * NB + part * VEC, g[u]);
        } else {
#pragma unroll
          for (int v = 0; v < VEC; ++v) g[u][v] = 0;
        }
      }
#pragma unroll
      for (int u = 0; u < KB; ++u) {
        const T c = p0 + u * ES < end ? table[e[u] >> col_bits] : static_cast<T>(0);
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[v] += c * g[u][v];
      }
    }
    if (ES > 1) {
#pragma unroll
      for (int o = LPR; o < G; o <<= 1)
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[v] += __shfl_xor_sync(group_mask, acc[v], o, G);
    }
    if (split == 0) {
      const T d = __ldcs(diag + r);
      T self[VEC];
      load16(z + r * NB + part * VEC, self);
      T o[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) o[v] = alpha * (acc[v] + d * self[v]) + beta * self[v];
      if (HAS_P) {
        T q[VEC];
        load16_rw(p + r * NB + part * VEC, q);
#pragma unroll
        for (int v = 0; v < VEC; ++v) o[v] += gamma * q[v];
      }
      store16(out + r * NB + part * VEC, o);
    }
  }
}

// Block action on the fly (matrix-free storage, real operators): one thread
// per row expands the adjoint products once and applies each transition to
// all NB columns of the row-major block, so the integer work of the expansion
// is shared by the NB vectors. In coordinates z = x / sqrt(R) the orbit ratio
// cancels: (S^-1 H S)[r, c] = conj(coefficient * amplitude) * phase.
// Epilogue as spmm_packed_kernel: out = alpha (S^-1 H S z) + beta z + gamma p.
template <typename S, typename T, int NB, bool HAS_P>
__global__ void __launch_bounds__(128) spmm_matrix_free_kernel(OpView<S> v, const T* __restrict__ z, const T* p,
                                                               T* out, T alpha, T beta, T gamma) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr int PARTS = NB / VEC;
  extern __shared__ Instance shared_inst[];
  const bool in_smem = v.n_inst <= kSmemInstances;
  if (in_smem)
    for (int k = threadIdx.x; k < v.n_inst; k += blockDim.x) shared_inst[k] = v.inst[k];
  __syncthreads();
  const Instance* inst = in_smem ? shared_inst : v.inst;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < v.dim; r += stride) {
    const S s = row_state(v, r);
    T acc[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) acc[j] = 0;
    double diag = 0.0;
    for (int k = 0; k < v.n_inst; ++k) {
      S t;
      double ar, ai;
      if (!apply_instance(inst[k], s, v.f, t, ar, ai)) continue;
      // real operators: conj(coefficient * amplitude) is real
      const double w = inst[k].cr * ar - inst[k].ci * ai;
      if (t == s) {
        diag += w;
        continue;
      }
      const Located L = locate(v, t);
      if (L.col < 0) continue;
      const T c = static_cast<T>(w * L.pr);
      const T* row = z + static_cast<uint64_t>(L.col) * NB;
#pragma unroll
      for (int q = 0; q < PARTS; ++q) {
        T g[VEC];
        load16(row + q * VEC, g);
#pragma unroll
        for (int u = 0; u < VEC; ++u) acc[q * VEC + u] += c * g[u];
      }
    }
    const T d = static_cast<T>(diag);
#pragma unroll
    for (int q = 0; q < PARTS; ++q) {
      T self[VEC], o[VEC];
      load16(z + r * NB + q * VEC, self);
#pragma unroll
      for (int u = 0; u < VEC; ++u) o[u] = alpha * (acc[q * VEC + u] + d * self[u]) + beta * self[u];
      if (HAS_P) {
        T pv[VEC];
        load16_rw(p + r * NB + q * VEC, pv);
#pragma unroll
        for (int u = 0; u < VEC; ++u) o[u] += gamma * pv[u];
      }
      store16(out + r * NB + q * VEC, o);
    }
  }
}

// Shapes of the block action tried by the autotuner: (ES, KB).
constexpr int kBlockShapes = 4;
constexpr int kBlockShapeES[kBlockShapes] = {1, 1, 2, 4};
constexpr int kBlockShapeKB[kBlockShapes] = {4, 8, 4, 2};
constexpr uint64_t kTuneMinRows = 1u << 20;  // smaller operators use shape 0 untimed

// xs = x / sqrt(R) elementwise (complex vectors scale both parts).
template <typename T>
__global__ void scale_by_orbit_kernel(uint64_t n, int comps, const uint16_t* __restrict__ orbits,
                                      const double* __restrict__ inv_sqrt, const T* __restrict__ x,
                                      T* __restrict__ xs) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n * comps; i += stride) {
    const uint64_t r = i / comps;
    xs[i] = __ldcs(x + i) * static_cast<T>(inv_sqrt[__ldcs(orbits + r)]);
  }
}

template <typename T>
__global__ void real_to_complex_kernel(uint64_t n, const T* __restrict__ x, T* __restrict__ out) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) {
    out[2 * i] = x[i];
    out[2 * i + 1] = 0;
  }
}

__global__ void convert_f64_to_f32_kernel(uint64_t n, const double* __restrict__ in, float* __restrict__ out) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = static_cast<float>(in[i]);
}

__global__ void real_part_kernel(uint64_t n, const double* __restrict__ in, double* __restrict__ out) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = in[2 * i];
}

int grid_for(uint64_t work, int threads, int per_sm = 8) {
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint64_t blocks = (work + threads - 1) / threads;
  uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
  return static_cast<int>(std::max<uint64_t>(1, std::min(blocks, cap)));
}

// apply_sector_shift (src/operator/mod.rs:2305-2351): one thread per source
// column; the forward products act on the column's representative, each
// target state is reduced into the target sector (index_transition,
// src/basis/mod.rs:1561-1580: sqrt(R_source / R_target) conj(phase), or 1
// when the target carries no symmetry) and added to its row atomically.
template <typename S>
__global__ void __launch_bounds__(128) sector_shift_kernel(OpView<S> src, OpView<S> tgt, const double* __restrict__ x,
                                                           double* __restrict__ y) {
  extern __shared__ Instance shared_inst[];
  const bool in_smem = src.n_inst <= kSmemInstances;
  if (in_smem)
    for (int k = threadIdx.x; k < src.n_inst; k += blockDim.x) shared_inst[k] = src.inst[k];
  __syncthreads();
  const Instance* inst = in_smem ? shared_inst : src.inst;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < src.dim; c += stride) {
    const double xr = x[2 * c], xi = x[2 * c + 1];
    if (hypot(xr, xi) <= 2.220446049250313e-16) continue;
    const S s = row_state(src, c);
    const int orbit = src.p.symmetric ? src.orbits[c] : 1;
    for (int k = 0; k < src.n_inst; ++k) {
      S t;
      double ar, ai;
      if (!apply_instance(inst[k], s, src.f, t, ar, ai)) continue;
      const Located L = locate(tgt, t);
      if (L.col < 0) continue;
      // coefficient * local amplitude * reduction amplitude
      double wr = inst[k].cr * ar - inst[k].ci * ai;
      double wi = inst[k].cr * ai + inst[k].ci * ar;
      if (tgt.p.symmetric) {
        const double ratio = tgt.inv_sqrt[257 + orbit] * tgt.inv_sqrt[L.orbit];
        const double pr = L.pr * ratio, pi = -L.pi * ratio;
        const double nr = wr * pr - wi * pi;
        wi = wr * pi + wi * pr;
        wr = nr;
      }
      atomicAdd(&y[2 * L.col], xr * wr - xi * wi);
      atomicAdd(&y[2 * L.col + 1], xr * wi + xi * wr);
    }
  }
}

template <typename S>
OpView<S> make_view(const SpinBasis& b, const DeviceBuffer& inst, int n_inst, const LocalFactors& f,
                    const DeviceBuffer& inv_sqrt) {
  OpView<S> v;
  v.p = b.params();
  v.mask = low_mask<S>(b.sites());
  v.states = static_cast<const S*>(b.states());
  v.orbits = b.orbits();
  v.dim = b.dim();
  v.direct = b.direct() ? 1 : 0;
  v.colex = b.colex() ? 1 : 0;
  v.binom = b.binomials();
  v.phase = b.phase_table();
  v.inv_sqrt = inv_sqrt.as<double>();
  v.inst = inst.as<Instance>();
  v.n_inst = n_inst;
  v.f = f;
  return v;
}

int read_flags(const DeviceBuffer& flags) {
  int h = 0;
  QMBED_CUDA(cudaMemcpy(&h, flags.get(), sizeof(int), cudaMemcpyDeviceToHost));
  return h;
}

}  // namespace

SpinOperator::SpinOperator(std::shared_ptr<SpinBasis> basis, const std::vector<TermDesc>& terms,
                           const OperatorChecks& checks, int storage)
    : basis_(std::move(basis)), storage_(storage) {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  build_instances(terms, checks);
  std::vector<double> table(2 * 257, 0.0);
  for (int r = 1; r <= 256; ++r) {
    table[r] = 1.0 / std::sqrt(static_cast<double>(r));
    table[257 + r] = std::sqrt(static_cast<double>(r));
  }
  table[257 + 0] = 0.0;
  inv_sqrt_.allocate(table.size() * sizeof(double));
  QMBED_CUDA(cudaMemcpy(inv_sqrt_.get(), table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice));
  // flip chains have real coefficients on symmetric flips and a real diagonal: Hermitian by construction
  if (checks.hermiticity && !flip_ && !check_hermitian()) raise(QMBED_NON_HERMITIAN, "");
  if (storage_ != kStorageMatrixFree) {
    if (dim() >= (1ULL << 32)) {
      storage_ = kStorageMatrixFree;  // columns do not fit 32 bits: keep the action matrix-free
    } else {
      assemble();
    }
  }
  // Matrix-free operators on a symmetry sector resolve their targets through
  // the basis's image table when it fits (built once, shared by every
  // operator on the basis); otherwise through the representative search.
  if (storage_ == kStorageMatrixFree && !flip_ && prog_.ok() && basis_->symmetric())
    basis_->build_image_table(false);
}

bool SpinOperator::launch_tile_action(const TileLaunch& l) const {
  if (lookup_mode_ == kLookupLegacy) return false;
  TileLaunch a = l;
  a.inv_sqrt = inv_sqrt_.as<double>();
  return launch_tile(*basis_, prog_, lookup_mode_, a);
}

void SpinOperator::apply_rows(int precision, uint64_t row0, uint64_t rows, const void* x, void* y,
                              cudaStream_t stream) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  const uint64_t n = dim();
  if (row0 > n || rows > n - row0) raise(QMBED_INVALID_OPTIONS, "row range outside the operator");
  if (!real_) raise(QMBED_UNSUPPORTED_BACKEND, "row slabs take real vectors of a real operator");
  if (storage_ != kStorageMatrixFree) raise(QMBED_UNSUPPORTED_BACKEND, "row slabs need matrix-free storage");
  if (rows == 0) return;
  TileLaunch tl;
  tl.precision = precision;
  tl.nb = 1;
  tl.x = x;
  tl.y = y;
  tl.stream = stream;
  tl.row0 = row0;
  tl.rows = rows;
  if (!launch_tile_action(tl))
    raise(QMBED_UNSUPPORTED_BACKEND, "row slabs need the tile kernel (u64 states, products on distinct sites)");
}

void SpinOperator::set_lookup(int mode) {
  if (mode < kLookupAuto || mode > kLookupTableGeneric) raise(QMBED_INVALID_OPTIONS, "unknown lookup mode");
  if (mode == kLookupTable || mode == kLookupTableGeneric) {
    if (!prog_.ok() || !basis_->symmetric())
      raise(QMBED_UNSUPPORTED_BACKEND, "image tables serve symmetry sectors of u64 states with a flip program");
    QMBED_CUDA(cudaSetDevice(basis_->device()));
    basis_->build_image_table(true);
  }
  lookup_mode_ = mode;
}

int SpinOperator::lookup_in_use() const {
  if (lookup_mode_ == kLookupLegacy || !prog_.ok() || basis_->words() != 1) return 3;
  if (!basis_->symmetric()) return 4;
  if (lookup_mode_ != kLookupSearch && basis_->image_table())
    return lookup_mode_ != kLookupTableGeneric && hop_kernel_applies(*basis_, prog_) ? 5 : 1;
  return 2;
}

void SpinOperator::build_instances(const std::vector<TermDesc>& terms, const OperatorChecks& checks) {
  const int sites = basis_->sites();
  const int norm = basis_->normalization();
  // Spin-1/2 local factors (SpinBasisBuilder::build, src/basis/mod.rs:1355-1376).
  factors_.z[0] = norm == kAngularMomentum ? -0.5 : -1.0;
  factors_.z[1] = norm == kAngularMomentum ? 0.5 : 1.0;
  factors_.raise = norm == kPauli ? 2.0 : 1.0;
  factors_.lower = norm == kPauli ? 2.0 : 1.0;
  factors_.xy_scale = norm == kPauliCartesian ? 1.0 : 0.5;

  std::vector<Instance> fwd, adj;
  bool real = basis_->real_phases();
  // (degree, expanded +/- string, sites) -> summed coefficient, for the
  // operator_sum_preserves_particle_sector check (src/operator/mod.rs:1963-2033).
  std::map<std::tuple<int, std::string, std::vector<int>>, C64> components;
  for (const TermDesc& term : terms) {
    const int arity = static_cast<int>(term.symbols.size());
    for (char c : term.symbols) {
      if (c != 'I' && c != 'z' && c != '+' && c != '-' && c != 'x' && c != 'y')
        raise(QMBED_INVALID_OPERATOR, std::string(1, c));
    }
    for (const CouplingDesc& coupling : term.couplings) {
      if (static_cast<int>(coupling.sites.size()) != arity)
        raise(QMBED_INVALID_COUPLING, "operator \"" + term.symbols + "\" has arity " + std::to_string(arity) +
                                          ", but a coupling has " + std::to_string(coupling.sites.size()) + " sites");
      if (!std::isfinite(coupling.coefficient.real()) || !std::isfinite(coupling.coefficient.imag()))
        raise(QMBED_INVALID_COUPLING, "coupling coefficients must be finite");
      if (arity > kMaxArity) raise(QMBED_UNSUPPORTED_BACKEND, "operator products act on at most 8 sites");
      for (int site : coupling.sites)
        if (site < 0 || site >= sites)
          raise(QMBED_INVALID_SITE, "site " + std::to_string(site) + " is outside a lattice with " +
                                        std::to_string(sites) + " sites");
      Instance f{}, a{};
      f.cr = coupling.coefficient.real();
      f.ci = coupling.coefficient.imag();
      a.cr = f.cr;
      a.ci = -f.ci;  // the adjoint product carries conj(c)
      f.n = a.n = arity;
      f.diagonal = 1;
      int n_y = 0;
      for (int q = 0; q < arity; ++q) {
        const char s = term.symbols[static_cast<size_t>(q)];
        f.sym[q] = s;
        f.site[q] = static_cast<uint8_t>(coupling.sites[static_cast<size_t>(q)]);
        const char dagger = s == '+' ? '-' : (s == '-' ? '+' : s);
        a.sym[arity - 1 - q] = dagger;
        a.site[arity - 1 - q] = f.site[q];
        if (s != 'I' && s != 'z') f.diagonal = 0;
        if (s == 'y') ++n_y;
      }
      a.diagonal = f.diagonal;
      // The amplitude of a product with n_y factors of y is i^{n_y} times a real number.
      C64 rotated = coupling.coefficient;
      for (int q = 0; q < n_y; ++q) rotated = C64(-rotated.imag(), rotated.real());  // exact multiply by i
      if (rotated.imag() != 0.0) real = false;
      fwd.push_back(f);
      adj.push_back(a);
      if (checks.particle_conservation && basis_->params().up >= 0) {
        std::vector<std::pair<std::string, C64>> expanded{{std::string(), C64(1.0, 0.0)}};
        int degree = 0;
        for (char s : term.symbols) {
          if (s == 'x' || s == 'y') {
            ++degree;
            std::vector<std::pair<std::string, C64>> next;
            for (auto& [prefix, coefficient] : expanded) {
              next.push_back({prefix + '+', coefficient * (s == 'x' ? C64(1, 0) : C64(0, -1))});
              next.push_back({prefix + '-', coefficient * (s == 'x' ? C64(1, 0) : C64(0, 1))});
            }
            expanded = std::move(next);
          } else {
            for (auto& item : expanded) item.first.push_back(s);
          }
        }
        for (auto& [op, coefficient] : expanded)
          components[{degree, op, coupling.sites}] += coupling.coefficient * coefficient;
      }
    }
  }
  if (checks.particle_conservation && basis_->params().up >= 0) {
    for (auto& [key, coefficient] : components) {
      if (std::abs(coefficient) <= 2.220446049250313e-16) continue;
      int change = 0;
      for (char s : std::get<1>(key)) change += s == '+' ? 1 : (s == '-' ? -1 : 0);
      const int target = basis_->params().up + change;
      if (!(target < 0 || target > sites || change == 0))
        raise(QMBED_INVALID_SECTOR, "operator sum does not preserve the selected particle sector");
    }
  }
  real_ = real;
  n_inst_ = static_cast<int>(adj.size());
  // Full-space chains whose products are z's (diagonal) or one x with
  // identities (a single bit flip) and real coefficients act through the
  // structured flip-chain kernels (matrix-free storage only).
  flip_.reset();
  if (storage_ == kStorageMatrixFree && basis_->direct() && !basis_->symmetric() && basis_->params().up < 0 &&
      sites <= 40 && factors_.raise == factors_.lower) {
    FlipChainDesc d;
    d.sites = sites;
    d.x_coefs.assign(static_cast<size_t>(sites), 0.0);
    std::map<uint64_t, double> diag;
    bool ok = true;
    for (const Instance& f : fwd) {
      if (f.ci != 0.0) {
        ok = false;
        break;
      }
      uint64_t zmask = 0, seen = 0;
      int flip_site = -1, nz = 0;
      for (int q = 0; q < f.n && ok; ++q) {
        if (f.sym[q] == 'I') continue;
        const uint64_t bit = 1ull << f.site[q];
        if (seen & bit) ok = false;
        seen |= bit;
        if (f.sym[q] == 'z') {
          zmask |= bit;
          ++nz;
        } else if (f.sym[q] == 'x' && flip_site < 0) {
          flip_site = f.site[q];
        } else {
          ok = false;
        }
      }
      if (!ok || (flip_site >= 0 && nz > 0)) {
        ok = false;
        break;
      }
      if (flip_site >= 0) d.x_coefs[static_cast<size_t>(flip_site)] += f.cr * factors_.raise * factors_.xy_scale;
      else diag[zmask] += f.cr * std::pow(factors_.z[1], nz);
    }
    if (ok && diag.size() <= 256) {
      for (const auto& [mask, c] : diag) {
        d.z_masks.push_back(mask);
        d.z_coefs.push_back(c);
      }
      flip_ = std::make_unique<FlipChain>(d);
      uint64_t flips = 0;
      for (double c : d.x_coefs) flips += c != 0.0 ? 1 : 0;
      nnz_off_ = flips * dim();
    }
  }
  if (basis_->words() == 1) prog_.upload(compile_flip_program(adj, factors_, sites, basis_->params().up >= 0));
  inst_adj_.allocate(std::max<size_t>(adj.size(), 1) * sizeof(Instance));
  inst_fwd_.allocate(std::max<size_t>(fwd.size(), 1) * sizeof(Instance));
  if (!adj.empty()) {
    QMBED_CUDA(cudaMemcpy(inst_adj_.get(), adj.data(), adj.size() * sizeof(Instance), cudaMemcpyHostToDevice));
    QMBED_CUDA(cudaMemcpy(inst_fwd_.get(), fwd.data(), fwd.size() * sizeof(Instance), cudaMemcpyHostToDevice));
  }
}

bool SpinOperator::check_hermitian() const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  if (dim() == 0 || n_inst_ == 0) return true;
  DeviceBuffer flags(sizeof(int));
  QMBED_CUDA(cudaMemset(flags.get(), 0, sizeof(int)));
  const int grid = grid_for(dim(), 128, 16);
  if (basis_->words() == 1) {
    auto v = make_view<uint64_t>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    hermitian_check_kernel<uint64_t><<<grid, 128>>>(v, inst_fwd_.as<Instance>(), flags.as<int>());
  } else {
    auto v = make_view<u128>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    hermitian_check_kernel<u128><<<grid, 128>>>(v, inst_fwd_.as<Instance>(), flags.as<int>());
  }
  QMBED_LAUNCH_CHECK();
  int h = read_flags(flags);
  if (h & kFlagRowOverflow)
    raise(QMBED_UNSUPPORTED_BACKEND, "more than 128 distinct transitions from one basis state");
  return (h & kFlagNonHermitian) == 0;
}

void SpinOperator::assemble() {
  auto start = std::chrono::steady_clock::now();
  const uint64_t n = dim();
  const int device_grid = grid_for(n, 128, 16);
  DeviceBuffer row_nnz(std::max<uint64_t>(n, 1) * sizeof(uint32_t));
  diag64_.allocate(std::max<uint64_t>(n, 1) * 2 * sizeof(double));
  DeviceBuffer dict(kDictSlots * sizeof(unsigned long long));
  DeviceBuffer flags(sizeof(int));
  QMBED_CUDA(cudaMemset(dict.get(), 0xff, kDictSlots * sizeof(unsigned long long)));
  QMBED_CUDA(cudaMemset(flags.get(), 0, sizeof(int)));
  const bool want_packed = real_ && storage_ == kStoragePacked;
  auto run_count = [&](auto tag) {
    using S = decltype(tag);
    auto v = make_view<S>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    assemble_count_kernel<S><<<device_grid, 128>>>(v, row_nnz.as<uint32_t>(), diag64_.as<double>(),
                                                   dict.as<unsigned long long>(), want_packed ? 1 : 0,
                                                   flags.as<int>());
  };
  if (basis_->words() == 1) run_count(uint64_t{});
  else run_count(u128{});
  QMBED_LAUNCH_CHECK();
  int h = read_flags(flags);
  if (h & kFlagRowOverflow) raise(QMBED_UNSUPPORTED_BACKEND, "more than 128 distinct transitions from one basis state");

  // Row pointer by exclusive scan of the row counts.
  nnz_off_ = exclusive_scan_counts(row_nnz.as<uint32_t>(), n, row_ptr_, &row_ptr64_);

  // Column bits and the value dictionary.
  col_bits_ = 1;
  while (col_bits_ < 32 && (1ULL << col_bits_) < std::max<uint64_t>(n, 2)) ++col_bits_;
  std::vector<double> codes_sorted;
  std::vector<int16_t> slot_codes(kDictSlots, -1);
  bool packed = want_packed && !(h & kFlagDictOverflow);
  if (packed) {
    std::vector<unsigned long long> keys(kDictSlots);
    QMBED_CUDA(cudaMemcpy(keys.data(), dict.get(), kDictSlots * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    std::vector<std::pair<double, int>> values;
    for (int slot = 0; slot < kDictSlots; ++slot) {
      if (keys[slot] == kDictEmpty) continue;
      double value;
      std::memcpy(&value, &keys[slot], sizeof(double));
      values.push_back({value, slot});
    }
    std::sort(values.begin(), values.end());
    const uint64_t code_capacity = col_bits_ >= 32 ? 1 : (1ULL << (32 - col_bits_));
    if (values.size() > static_cast<size_t>(kMaxCodes) || values.size() > code_capacity || values.empty()) {
      packed = values.empty() && nnz_off_ == 0;  // an all-diagonal operator needs no codes
      if (values.empty()) codes_sorted.push_back(0.0);
    } else {
      for (size_t i = 0; i < values.size(); ++i) {
        codes_sorted.push_back(values[i].first);
        slot_codes[values[i].second] = static_cast<int16_t>(i);
      }
    }
  }
  n_codes_ = static_cast<int>(codes_sorted.size());
  storage_ = packed ? kStoragePacked : kStorageWide;
  entries_.allocate(std::max<uint64_t>(nnz_off_, 1) * sizeof(uint32_t));
  DeviceBuffer slot_dev(kDictSlots * sizeof(int16_t));
  if (packed) {
    QMBED_CUDA(cudaMemcpy(slot_dev.get(), slot_codes.data(), kDictSlots * sizeof(int16_t), cudaMemcpyHostToDevice));
    code_table_.allocate(std::max<size_t>(codes_sorted.size(), 1) * sizeof(double));
    if (!codes_sorted.empty())
      QMBED_CUDA(cudaMemcpy(code_table_.get(), codes_sorted.data(), codes_sorted.size() * sizeof(double),
                            cudaMemcpyHostToDevice));
  } else {
    values64_.allocate(std::max<uint64_t>(nnz_off_, 1) * 2 * sizeof(double));
  }
  auto run_fill = [&](auto tag) {
    using S = decltype(tag);
    auto v = make_view<S>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    if (row_ptr64_)
      assemble_fill_kernel<S, uint64_t><<<device_grid, 128>>>(
          v, row_ptr_.as<uint64_t>(), entries_.as<uint32_t>(), packed ? nullptr : values64_.as<double>(),
          dict.as<unsigned long long>(), packed ? slot_dev.as<int16_t>() : nullptr, packed ? col_bits_ : 32,
          flags.as<int>());
    else
      assemble_fill_kernel<S, uint32_t><<<device_grid, 128>>>(
          v, row_ptr_.as<uint32_t>(), entries_.as<uint32_t>(), packed ? nullptr : values64_.as<double>(),
          dict.as<unsigned long long>(), packed ? slot_dev.as<int16_t>() : nullptr, packed ? col_bits_ : 32,
          flags.as<int>());
  };
  if (basis_->words() == 1) run_fill(uint64_t{});
  else run_fill(u128{});
  QMBED_LAUNCH_CHECK();
  h = read_flags(flags);
  if (h & kFlagDictOverflow) raise(QMBED_INTERNAL_STATE, "value dictionary lookup failed during assembly");
  if (!packed) col_bits_ = 32;

  // Precision copies: FP32 diagonal (and values), real diagonal for real operators.
  const uint64_t diag_len = 2 * n;
  if (real_) {
    DeviceBuffer real_diag(std::max<uint64_t>(n, 1) * sizeof(double));
    real_part_kernel<<<grid_for(n, 256), 256>>>(n, diag64_.as<double>(), real_diag.as<double>());
    QMBED_LAUNCH_CHECK();
    diag64_ = std::move(real_diag);
    diag32_.allocate(std::max<uint64_t>(n, 1) * sizeof(float));
    convert_f64_to_f32_kernel<<<grid_for(n, 256), 256>>>(n, diag64_.as<double>(), diag32_.as<float>());
  } else {
    diag32_.allocate(std::max<uint64_t>(diag_len, 1) * sizeof(float));
    convert_f64_to_f32_kernel<<<grid_for(diag_len, 256), 256>>>(diag_len, diag64_.as<double>(), diag32_.as<float>());
  }
  QMBED_LAUNCH_CHECK();
  if (!packed && nnz_off_ > 0) {
    values32_.allocate(nnz_off_ * 2 * sizeof(float));
    convert_f64_to_f32_kernel<<<grid_for(2 * nnz_off_, 256), 256>>>(2 * nnz_off_, values64_.as<double>(),
                                                                     values32_.as<float>());
    QMBED_LAUNCH_CHECK();
  }
  QMBED_CUDA(cudaDeviceSynchronize());
  assembly_seconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

void SpinOperator::ensure_scratch(int precision, bool complex_vectors) const {
  const size_t bytes = static_cast<size_t>(dim()) * (complex_vectors ? 2 : 1) * (precision == kFP64 ? 8 : 4);
  if (scaled_bytes_ < bytes) {
    scaled_x_.allocate(bytes);
    scaled_bytes_ = bytes;
  }
}

void SpinOperator::apply(int precision, bool complex_vectors, const void* x, void* y, cudaStream_t stream,
                         bool force_matrix_free) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  const uint64_t n = dim();
  if (n == 0) return;
  if (!real_ && !complex_vectors)
    raise(QMBED_UNSUPPORTED_BACKEND, "real action requires an operator with real-valued storage");
  const bool cplx = complex_vectors;
  if (flip_ && !force_matrix_free) {
    flip_->apply(precision, cplx, x, y, nullptr, nullptr, FlipStep{}, stream);
    return;
  }
  // Wide rows of a real operator keep a real diagonal: complex vectors take the matrix-free path.
  if (real_ && cplx && storage_ == kStorageWide) force_matrix_free = true;
  if (storage_ == kStorageMatrixFree || force_matrix_free) {
    TileLaunch tl;
    tl.precision = precision;
    tl.nb = 1;
    tl.complex_vectors = cplx;
    tl.x = x;
    tl.y = y;
    tl.stream = stream;
    if (launch_tile_action(tl)) return;
    const int grid = grid_for(n, 256, 8);
    const size_t smem = n_inst_ <= kSmemInstances ? static_cast<size_t>(n_inst_) * sizeof(Instance) : 0;
    auto launch = [&](auto stag, auto ttag, auto ctag) {
      using S = decltype(stag);
      using T = decltype(ttag);
      constexpr bool C = decltype(ctag)::value;
      auto v = make_view<S>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
      auto kernel = hv_matrix_free_kernel<S, T, C>;
      if (smem > 48 * 1024) QMBED_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                            static_cast<int>(smem)));
      kernel<<<grid, 256, smem, stream>>>(v, static_cast<const T*>(x), static_cast<T*>(y));
    };
    using True = std::true_type;
    using False = std::false_type;
    if (basis_->words() == 1) {
      if (precision == kFP64) cplx ? launch(uint64_t{}, double{}, True{}) : launch(uint64_t{}, double{}, False{});
      else cplx ? launch(uint64_t{}, float{}, True{}) : launch(uint64_t{}, float{}, False{});
    } else {
      if (precision == kFP64) cplx ? launch(u128{}, double{}, True{}) : launch(u128{}, double{}, False{});
      else cplx ? launch(u128{}, float{}, True{}) : launch(u128{}, float{}, False{});
    }
    QMBED_LAUNCH_CHECK();
    return;
  }
  // Stored rows.
  const bool scaled = basis_->symmetric();
  const void* xs = x;
  if (scaled) {
    ensure_scratch(precision, cplx);
    const int comps = cplx ? 2 : 1;
    const int grid = grid_for(n * comps, 256, 16);
    if (precision == kFP64)
      scale_by_orbit_kernel<double><<<grid, 256, 0, stream>>>(n, comps, basis_->orbits(), inv_sqrt_.as<double>(),
                                                               static_cast<const double*>(x), scaled_x_.as<double>());
    else
      scale_by_orbit_kernel<float><<<grid, 256, 0, stream>>>(n, comps, basis_->orbits(), inv_sqrt_.as<double>(),
                                                              static_cast<const float*>(x), scaled_x_.as<float>());
    QMBED_LAUNCH_CHECK();
    xs = scaled_x_.get();
  }
  constexpr int kLanes = 4;
  const int grid = grid_for(n * kLanes, 256, 8);
  if (storage_ == kStoragePacked) {
    auto launch = [&](auto ttag, auto itag, auto stag) {
      using T = decltype(ttag);
      using I = decltype(itag);
      constexpr bool SC = decltype(stag)::value;
      const T* diag = precision == kFP64 ? reinterpret_cast<const T*>(diag64_.get()) : reinterpret_cast<const T*>(diag32_.get());
      auto kernel = cplx ? spmv_packed_kernel<T, I, SC, kLanes, true> : spmv_packed_kernel<T, I, SC, kLanes, false>;
      kernel<<<grid, 256, 0, stream>>>(n, row_ptr_.as<I>(), entries_.as<uint32_t>(), col_bits_,
                                       code_table_.as<double>(), n_codes_, diag, basis_->orbits(),
                                       inv_sqrt_.as<double>(), static_cast<const T*>(xs), static_cast<const T*>(x),
                                       static_cast<T*>(y));
    };
    using True = std::true_type;
    using False = std::false_type;
    if (precision == kFP64) {
      if (row_ptr64_) scaled ? launch(double{}, uint64_t{}, True{}) : launch(double{}, uint64_t{}, False{});
      else scaled ? launch(double{}, uint32_t{}, True{}) : launch(double{}, uint32_t{}, False{});
    } else {
      if (row_ptr64_) scaled ? launch(float{}, uint64_t{}, True{}) : launch(float{}, uint64_t{}, False{});
      else scaled ? launch(float{}, uint32_t{}, True{}) : launch(float{}, uint32_t{}, False{});
    }
    QMBED_LAUNCH_CHECK();
    return;
  }
  // Wide storage: explicit (interleaved complex) values.
  const void* xin = x;
  void* yout = y;
  auto launch = [&](auto ttag, auto itag, auto stag) {
    using T = decltype(ttag);
    using I = decltype(itag);
    constexpr bool SC = decltype(stag)::value;
    auto kernel = cplx ? spmv_wide_kernel<T, I, SC, kLanes, true> : spmv_wide_kernel<T, I, SC, kLanes, false>;
    const T* diag = precision == kFP64 ? reinterpret_cast<const T*>(diag64_.get()) : reinterpret_cast<const T*>(diag32_.get());
    const T* vals = precision == kFP64 ? reinterpret_cast<const T*>(values64_.get()) : reinterpret_cast<const T*>(values32_.get());
    kernel<<<grid, 256, 0, stream>>>(n, row_ptr_.as<I>(), entries_.as<uint32_t>(), vals,
                                                                 diag, basis_->orbits(), inv_sqrt_.as<double>(),
                                                                 static_cast<const T*>(xs), static_cast<const T*>(xin),
                                                                 static_cast<T*>(yout));
  };
  using True = std::true_type;
  using False = std::false_type;
  if (precision == kFP64) {
    if (row_ptr64_) scaled ? launch(double{}, uint64_t{}, True{}) : launch(double{}, uint64_t{}, False{});
    else scaled ? launch(double{}, uint32_t{}, True{}) : launch(double{}, uint32_t{}, False{});
  } else {
    if (row_ptr64_) scaled ? launch(float{}, uint64_t{}, True{}) : launch(float{}, uint64_t{}, False{});
    else scaled ? launch(float{}, uint32_t{}, True{}) : launch(float{}, uint32_t{}, False{});
  }
  QMBED_LAUNCH_CHECK();
}

void SpinOperator::apply_with_scratch(int precision, bool complex_vectors, const void* x, void* y,
                                      cudaStream_t stream, void* scratch, size_t scratch_bytes) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  const uint64_t n = dim();
  if (n == 0) return;
  const bool cplx = complex_vectors;
  // wide rows of a real operator with complex vectors run matrix-free (their diagonal is real)
  const bool stored_symmetric = storage_ != kStorageMatrixFree && basis_->symmetric() &&
                                !(real_ && cplx && storage_ == kStorageWide);
  if (!stored_symmetric) {
    // These paths hold no scaled vector. Flip chains and wide rows of a real
    // operator with complex vectors take the on-the-fly expansion, whose
    // kernels need no work buffer (the flip-chain kernels would allocate their
    // diagonal tables on first use).
    apply(precision, complex_vectors, x, y, stream, flip_ != nullptr || (real_ && cplx && storage_ == kStorageWide));
    return;
  }
  if (!real_ && !cplx) raise(QMBED_UNSUPPORTED_BACKEND, "real action requires an operator with real-valued storage");
  const int comps = cplx ? 2 : 1;
  const size_t need = static_cast<size_t>(n) * comps * (precision == kFP64 ? 8 : 4);
  if (need > scratch_bytes)
    raise(QMBED_DIMENSION_MISMATCH, "symmetry sectors with stored rows take vectors of at most " +
                                        std::to_string(scratch_bytes) + " bytes here; this one has " +
                                        std::to_string(need));
  {
    const int grid = grid_for(n * comps, 256, 16);
    if (precision == kFP64)
      scale_by_orbit_kernel<double><<<grid, 256, 0, stream>>>(n, comps, basis_->orbits(), inv_sqrt_.as<double>(),
                                                               static_cast<const double*>(x),
                                                               static_cast<double*>(scratch));
    else
      scale_by_orbit_kernel<float><<<grid, 256, 0, stream>>>(n, comps, basis_->orbits(), inv_sqrt_.as<double>(),
                                                              static_cast<const float*>(x),
                                                              static_cast<float*>(scratch));
    QMBED_LAUNCH_CHECK();
  }
  const void* xs = scratch;
  constexpr int kLanes = 4;
  const int grid = grid_for(n * kLanes, 256, 8);
  using True = std::true_type;
  if (storage_ == kStoragePacked) {
    auto launch = [&](auto ttag, auto itag) {
      using T = decltype(ttag);
      using I = decltype(itag);
      const T* diag = precision == kFP64 ? reinterpret_cast<const T*>(diag64_.get()) : reinterpret_cast<const T*>(diag32_.get());
      auto kernel = cplx ? spmv_packed_kernel<T, I, True::value, kLanes, true>
                         : spmv_packed_kernel<T, I, True::value, kLanes, false>;
      kernel<<<grid, 256, 0, stream>>>(n, row_ptr_.as<I>(), entries_.as<uint32_t>(), col_bits_,
                                       code_table_.as<double>(), n_codes_, diag, basis_->orbits(),
                                       inv_sqrt_.as<double>(), static_cast<const T*>(xs), static_cast<const T*>(x),
                                       static_cast<T*>(y));
    };
    if (precision == kFP64) row_ptr64_ ? launch(double{}, uint64_t{}) : launch(double{}, uint32_t{});
    else row_ptr64_ ? launch(float{}, uint64_t{}) : launch(float{}, uint32_t{});
    QMBED_LAUNCH_CHECK();
    return;
  }
  auto launch = [&](auto ttag, auto itag) {
    using T = decltype(ttag);
    using I = decltype(itag);
    auto kernel = cplx ? spmv_wide_kernel<T, I, True::value, kLanes, true> : spmv_wide_kernel<T, I, True::value, kLanes, false>;
    const T* diag = precision == kFP64 ? reinterpret_cast<const T*>(diag64_.get()) : reinterpret_cast<const T*>(diag32_.get());
    const T* vals = precision == kFP64 ? reinterpret_cast<const T*>(values64_.get()) : reinterpret_cast<const T*>(values32_.get());
    kernel<<<grid, 256, 0, stream>>>(n, row_ptr_.as<I>(), entries_.as<uint32_t>(), vals, diag, basis_->orbits(),
                                     inv_sqrt_.as<double>(), static_cast<const T*>(xs), static_cast<const T*>(x),
                                     static_cast<T*>(y));
  };
  if (precision == kFP64) row_ptr64_ ? launch(double{}, uint64_t{}) : launch(double{}, uint32_t{});
  else row_ptr64_ ? launch(float{}, uint64_t{}) : launch(float{}, uint32_t{});
  QMBED_LAUNCH_CHECK();
}

SpinOperator::ExplicitRows SpinOperator::explicit_rows() const {
  if (storage_ != kStorageWide) raise(QMBED_UNSUPPORTED_BACKEND, "the operator does not hold rows with explicit values");
  ExplicitRows r;
  r.n = dim();
  r.row_ptr64 = row_ptr64_;
  r.row_ptr = row_ptr_.get();
  r.cols = entries_.as<uint32_t>();
  r.values = values64_.as<double>();
  r.diag = diag64_.as<double>();
  r.diag_complex = !real_;
  return r;
}

bool SpinOperator::supports_block() const {
  return real_ && (storage_ == kStoragePacked || storage_ == kStorageMatrixFree);
}

void SpinOperator::launch_block_matrix_free(int precision, int nb, const void* z, const void* p, void* out,
                                            double alpha, double beta, double gamma, cudaStream_t stream) const {
  TileLaunch tl;
  tl.precision = precision;
  tl.nb = nb;
  tl.x = z;
  tl.p = p;
  tl.y = out;
  tl.alpha = alpha;
  tl.beta = beta;
  tl.gamma = gamma;
  tl.stream = stream;
  if (launch_tile_action(tl)) return;
  const int grid = grid_for(dim(), 128, 16);
  const size_t smem = n_inst_ <= kSmemInstances ? static_cast<size_t>(n_inst_) * sizeof(Instance) : 0;
  auto launch = [&](auto stag, auto ttag, auto nbtag, auto ptag) {
    using S = decltype(stag);
    using T = decltype(ttag);
    constexpr int NB = decltype(nbtag)::value;
    constexpr bool HP = decltype(ptag)::value;
    auto v = make_view<S>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    spmm_matrix_free_kernel<S, T, NB, HP><<<grid, 128, smem, stream>>>(
        v, static_cast<const T*>(z), static_cast<const T*>(p), static_cast<T*>(out), static_cast<T>(alpha),
        static_cast<T>(beta), static_cast<T>(gamma));
  };
  auto by_p = [&](auto stag, auto ttag, auto nbtag) {
    if (p) launch(stag, ttag, nbtag, std::true_type{});
    else launch(stag, ttag, nbtag, std::false_type{});
  };
  auto by_nb = [&](auto stag, auto ttag) {
    if (nb == 8) by_p(stag, ttag, std::integral_constant<int, 8>{});
    else by_p(stag, ttag, std::integral_constant<int, 16>{});
  };
  auto by_t = [&](auto stag) {
    if (precision == kFP64) by_nb(stag, double{});
    else by_nb(stag, float{});
  };
  if (basis_->words() == 1) by_t(uint64_t{});
  else by_t(u128{});
  QMBED_LAUNCH_CHECK();
}

void SpinOperator::launch_block(int shape, int precision, int nb, const void* z, const void* p, void* out,
                                double alpha, double beta, double gamma, cudaStream_t stream) const {
  const uint64_t n = dim();
  auto launch = [&](auto ttag, auto itag, auto nbtag, auto ptag, auto estag, auto kbtag) {
    using T = decltype(ttag);
    using I = decltype(itag);
    constexpr int NB = decltype(nbtag)::value;
    constexpr bool HP = decltype(ptag)::value;
    constexpr int ES = decltype(estag)::value;
    constexpr int KB = decltype(kbtag)::value;
    constexpr int G = NB / (16 / static_cast<int>(sizeof(T))) * ES;
    const T* diag = precision == kFP64 ? reinterpret_cast<const T*>(diag64_.get()) : reinterpret_cast<const T*>(diag32_.get());
    const int grid = grid_for(n * G, 256, 8);
    spmm_packed_kernel<T, I, NB, HP, ES, KB><<<grid, 256, 0, stream>>>(
        n, row_ptr_.as<I>(), entries_.as<uint32_t>(), col_bits_, code_table_.as<double>(), n_codes_, diag,
        static_cast<const T*>(z), static_cast<const T*>(p), static_cast<T*>(out), static_cast<T>(alpha),
        static_cast<T>(beta), static_cast<T>(gamma));
  };
  using NB8 = std::integral_constant<int, 8>;
  using NB16 = std::integral_constant<int, 16>;
  auto by_shape = [&](auto ttag, auto itag, auto nbtag, auto ptag) {
    switch (shape) {
      case 1: launch(ttag, itag, nbtag, ptag, std::integral_constant<int, 1>{}, std::integral_constant<int, 8>{}); break;
      case 2: launch(ttag, itag, nbtag, ptag, std::integral_constant<int, 2>{}, std::integral_constant<int, 4>{}); break;
      case 3: launch(ttag, itag, nbtag, ptag, std::integral_constant<int, 4>{}, std::integral_constant<int, 2>{}); break;
      default: launch(ttag, itag, nbtag, ptag, std::integral_constant<int, 1>{}, std::integral_constant<int, 4>{}); break;
    }
  };
  auto by_p = [&](auto ttag, auto itag, auto nbtag) {
    if (p) by_shape(ttag, itag, nbtag, std::true_type{});
    else by_shape(ttag, itag, nbtag, std::false_type{});
  };
  auto by_nb = [&](auto ttag, auto itag) {
    if (nb == 8) by_p(ttag, itag, NB8{});
    else by_p(ttag, itag, NB16{});
  };
  if (precision == kFP64) row_ptr64_ ? by_nb(double{}, uint64_t{}) : by_nb(double{}, uint32_t{});
  else row_ptr64_ ? by_nb(float{}, uint64_t{}) : by_nb(float{}, uint32_t{});
  QMBED_LAUNCH_CHECK();
}

// Autotuner: the first call of each (precision, width, with/without p) on an
// operator of at least kTuneMinRows rows times every shape on the caller's
// inputs (output to a scratch block, so the caller's p is untouched) and keeps
// the fastest; later calls reuse it.
int SpinOperator::block_shape(int precision, int nb, const void* z, const void* p, double alpha, double beta,
                              double gamma, cudaStream_t stream) const {
  // QMBED_BLOCK_SHAPE=<index> pins a shape (for tests of every shape)
  const char* forced = std::getenv("QMBED_BLOCK_SHAPE");
  if (forced && forced[0] >= '0' && forced[0] < '0' + kBlockShapes && forced[1] == '\0') return forced[0] - '0';
  const int key = precision * 1000 + nb * 10 + (p ? 1 : 0);
  std::lock_guard<std::mutex> lock(tune_mu_);
  auto it = block_shapes_.find(key);
  if (it != block_shapes_.end()) return it->second;
  const uint64_t n = dim();
  int best = 0;
  if (n >= kTuneMinRows) {
    DeviceBuffer scratch(static_cast<size_t>(n) * nb * (precision == kFP64 ? 8 : 4));
    cudaEvent_t start, stop;
    QMBED_CUDA(cudaEventCreate(&start));
    QMBED_CUDA(cudaEventCreate(&stop));
    float best_ms = 0.0f;
    for (int shape = 0; shape < kBlockShapes; ++shape) {
      launch_block(shape, precision, nb, z, p, scratch.get(), alpha, beta, gamma, stream);  // warm
      QMBED_CUDA(cudaEventRecord(start, stream));
      for (int rep = 0; rep < 3; ++rep)
        launch_block(shape, precision, nb, z, p, scratch.get(), alpha, beta, gamma, stream);
      QMBED_CUDA(cudaEventRecord(stop, stream));
      QMBED_CUDA(cudaEventSynchronize(stop));
      float ms = 0.0f;
      QMBED_CUDA(cudaEventElapsedTime(&ms, start, stop));
      if (shape == 0 || ms < best_ms) {
        best_ms = ms;
        best = shape;
      }
      const char* trace = std::getenv("QMBED_FILTER_TRACE");
      if (trace && trace[0] == '1')
        std::fprintf(stderr, "[block tune] fp%d nb=%d p=%d shape ES=%d KB=%d: %.3f ms\n", precision, nb, p ? 1 : 0,
                     kBlockShapeES[shape], kBlockShapeKB[shape], ms / 3.0f);
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
  }
  block_shapes_[key] = best;
  return best;
}

int SpinOperator::tuned_block_shape(int precision, int nb, bool with_p) const {
  std::lock_guard<std::mutex> lock(tune_mu_);
  auto it = block_shapes_.find(precision * 1000 + nb * 10 + (with_p ? 1 : 0));
  return it == block_shapes_.end() ? -1 : it->second;
}

void SpinOperator::apply_block(int precision, int nb, const void* z, const void* p, void* out, double alpha,
                               double beta, double gamma, cudaStream_t stream) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  if (!supports_block()) raise(QMBED_UNSUPPORTED_BACKEND, "block action needs a real operator with packed rows or matrix-free storage");
  if (nb != 8 && nb != 16) raise(QMBED_INVALID_OPTIONS, "block width must be 8 or 16");
  if (dim() == 0) return;
  if (storage_ == kStorageMatrixFree) {
    launch_block_matrix_free(precision, nb, z, p, out, alpha, beta, gamma, stream);
    return;
  }
  const int shape = block_shape(precision, nb, z, p, alpha, beta, gamma, stream);
  launch_block(shape, precision, nb, z, p, out, alpha, beta, gamma, stream);
}

void SpinOperator::apply_shift(const SpinBasis& target, const double* x, double* y, cudaStream_t stream) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  if (target.sites() != basis_->sites() || target.words() != basis_->words() ||
      target.device() != basis_->device())
    raise(QMBED_DIMENSION_MISMATCH, "sector-shift state dimensions do not match source and target bases");
  QMBED_CUDA(cudaMemsetAsync(y, 0, std::max<uint64_t>(target.dim(), 1) * 16, stream));
  if (dim() == 0 || target.dim() == 0 || n_inst_ == 0) return;
  const int grid = grid_for(dim(), 128, 16);
  const size_t smem = n_inst_ <= kSmemInstances ? static_cast<size_t>(n_inst_) * sizeof(Instance) : 0;
  DeviceBuffer unused;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    auto src = make_view<S>(*basis_, inst_fwd_, n_inst_, factors_, inv_sqrt_);
    auto tgt = make_view<S>(target, unused, 0, factors_, inv_sqrt_);
    sector_shift_kernel<S><<<grid, 128, smem, stream>>>(src, tgt, x, y);
  };
  if (basis_->words() == 1) run(uint64_t{});
  else run(u128{});
  QMBED_LAUNCH_CHECK();
}

void SpinOperator::export_csr(std::vector<uint64_t>& row_ptr, std::vector<uint32_t>& cols,
                              std::vector<C64>& values) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  if (storage_ == kStorageMatrixFree) raise(QMBED_UNSUPPORTED_BACKEND, "matrix-free operators hold no stored rows");
  const uint64_t n = dim();
  row_ptr.resize(n + 1);
  if (row_ptr64_) {
    QMBED_CUDA(cudaMemcpy(row_ptr.data(), row_ptr_.get(), (n + 1) * 8, cudaMemcpyDeviceToHost));
  } else {
    std::vector<uint32_t> tmp(n + 1);
    QMBED_CUDA(cudaMemcpy(tmp.data(), row_ptr_.get(), (n + 1) * 4, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i <= n; ++i) row_ptr[i] = tmp[i];
  }
  std::vector<uint32_t> entries(nnz_off_);
  if (nnz_off_) QMBED_CUDA(cudaMemcpy(entries.data(), entries_.get(), nnz_off_ * 4, cudaMemcpyDeviceToHost));
  std::vector<double> diag(real_ ? n : 2 * n);
  QMBED_CUDA(cudaMemcpy(diag.data(), diag64_.get(), diag.size() * 8, cudaMemcpyDeviceToHost));
  std::vector<double> codes(n_codes_);
  if (storage_ == kStoragePacked && n_codes_)
    QMBED_CUDA(cudaMemcpy(codes.data(), code_table_.get(), n_codes_ * 8, cudaMemcpyDeviceToHost));
  std::vector<double> vals;
  if (storage_ == kStorageWide && nnz_off_) {
    vals.resize(2 * nnz_off_);
    QMBED_CUDA(cudaMemcpy(vals.data(), values64_.get(), vals.size() * 8, cudaMemcpyDeviceToHost));
  }
  std::vector<uint16_t> orbits(n, 1);
  if (basis_->symmetric()) QMBED_CUDA(cudaMemcpy(orbits.data(), basis_->orbits(), n * 2, cudaMemcpyDeviceToHost));
  // Full rows including the diagonal, in column order, with the orbit ratio applied.
  std::vector<uint64_t> out_ptr(n + 1, 0);
  cols.clear();
  values.clear();
  const uint32_t mask = col_bits_ >= 32 ? 0xffffffffu : ((1u << col_bits_) - 1u);
  for (uint64_t r = 0; r < n; ++r) {
    std::vector<std::pair<uint32_t, C64>> row;
    C64 d = real_ ? C64(diag[r], 0.0) : C64(diag[2 * r], diag[2 * r + 1]);
    if (std::abs(d) > 0.0) row.push_back({static_cast<uint32_t>(r), d});
    for (uint64_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
      uint32_t c, code;
      C64 w;
      if (storage_ == kStoragePacked) {
        c = entries[p] & mask;
        code = entries[p] >> col_bits_;
        w = C64(codes[code], 0.0);
      } else {
        c = entries[p];
        w = C64(vals[2 * p], vals[2 * p + 1]);
      }
      double ratio = std::sqrt(static_cast<double>(orbits[r])) / std::sqrt(static_cast<double>(orbits[c]));
      row.push_back({c, w * ratio});
    }
    std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& e : row) {
      cols.push_back(e.first);
      values.push_back(e.second);
    }
    out_ptr[r + 1] = cols.size();
  }
  row_ptr = std::move(out_ptr);
}

void SpinOperator::trace_and_one_norm(C64* shift, double* one_norm) const {
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  const uint64_t n = dim();
  if (n == 0) {
    *shift = C64(0.0, 0.0);
    *one_norm = 0.0;
    return;
  }
  DeviceBuffer diag(n * 2 * sizeof(double)), offsum(n * sizeof(double)), flags(sizeof(int));
  QMBED_CUDA(cudaMemset(flags.get(), 0, sizeof(int)));
  const int grid = grid_for(n, 128, 16);
  if (basis_->words() == 1) {
    auto v = make_view<uint64_t>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    column_norm_kernel<uint64_t><<<grid, 128>>>(v, inst_fwd_.as<Instance>(), diag.as<double>(), offsum.as<double>(),
                                                flags.as<int>());
  } else {
    auto v = make_view<u128>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    column_norm_kernel<u128><<<grid, 128>>>(v, inst_fwd_.as<Instance>(), diag.as<double>(), offsum.as<double>(),
                                            flags.as<int>());
  }
  QMBED_LAUNCH_CHECK();
  if (read_flags(flags) & kFlagRowOverflow)
    raise(QMBED_UNSUPPORTED_BACKEND, "more than 128 distinct transitions from one basis state");
  C64 trace = device_sum_complex(diag.as<double>(), n);
  *shift = trace / static_cast<double>(n);
  *one_norm = device_max_shifted_column(diag.as<double>(), offsum.as<double>(), n, *shift);
}

uint64_t SpinOperator::count_offdiag() const {
  if (counted_nnz_ != ~0ull) return counted_nnz_;
  QMBED_CUDA(cudaSetDevice(basis_->device()));
  const uint64_t n = dim();
  if (n == 0) return counted_nnz_ = 0;
  DeviceBuffer row_nnz(n * sizeof(uint32_t)), diag(n * 2 * sizeof(double)), flags(sizeof(int));
  QMBED_CUDA(cudaMemset(flags.get(), 0, sizeof(int)));
  auto run = [&](auto tag) {
    using S = decltype(tag);
    auto v = make_view<S>(*basis_, inst_adj_, n_inst_, factors_, inv_sqrt_);
    assemble_count_kernel<S><<<grid_for(n, 128, 16), 128>>>(v, row_nnz.as<uint32_t>(), diag.as<double>(), nullptr, 0,
                                                             flags.as<int>());
  };
  if (basis_->words() == 1) run(uint64_t{});
  else run(u128{});
  QMBED_LAUNCH_CHECK();
  DeviceBuffer row_ptr;
  bool wide = false;
  counted_nnz_ = exclusive_scan_counts(row_nnz.as<uint32_t>(), n, row_ptr, &wide);
  return counted_nnz_;
}

double SpinOperator::operand_bytes(int precision, bool complex_vectors) const {
  const double s = (precision == kFP64 ? 8.0 : 4.0) * (complex_vectors ? 2.0 : 1.0);
  const double b_state = basis_->direct() ? 0.0 : 8.0 * basis_->words();
  const double n = static_cast<double>(dim());
  uint64_t nnz = nnz_off_;
  if (storage_ == kStorageMatrixFree && !flip_) nnz = count_offdiag();
  return n * (b_state + s) + (n + static_cast<double>(nnz)) * s;
}

}  // namespace qmbed
