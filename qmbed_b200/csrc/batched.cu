// Batched Lanczos over sectors x scan points in one persistent launch.
//
// Every (sector s, point p) pair is an independent Hermitian problem
// H(s, p) = sum_k c_k(p) A_k(s) whose lowest eigenvalues are wanted (the
// reference calls eigsh once per pair, src/solve/mod.rs:2335-2350). Here all
// pairs advance together: one column per pair in row-major blocks (rows of
// sector s) x (points), so one pass applies every sector's operator to every
// point, and the gather of a column reads all points of that row as one
// contiguous 512-byte or 1-KB line. The rows of all sectors are concatenated
// and each warp finds its sector by binary search, so sectors of uneven
// dimension share the launch.
//
// Execution: a cooperative kernel runs a chunk of Lanczos steps; its phases
// (apply, alpha, update, beta, scale) are separated by a grid barrier whose
// spin is bounded (on time-out every block records the error and returns).
// A chunk is [persistent kernel, convergence check, status copy]; it is
// captured once in a CUDA graph and replayed until every pair has converged.
// The step counter lives in device memory, so the graph's arguments never
// change.
//
// Method: plain three-term Lanczos without reorthogonalisation, FP64 vectors
// and recurrences, orbit-scaled coordinates z = x / sqrt(R) with R-weighted
// inner products. A pair stops when the residual estimates |beta_m s_m| of
// its lowest Ritz values (copies from lost orthogonality counted once) are
// below 0.5 tol max(|theta|, 1); a sector's rows leave the recurrence once all
// its pairs have stopped. A second pass repeats the identical
// recurrence and accumulates the Ritz vectors of the lowest candidates; one
// FP64 application then gives every candidate's true residual
// ||H v - theta v|| / ||v|| (the reference's acceptance test, src/solve/mod.rs:
// 1252-1263) and the overlaps that decide which close Ritz values are copies
// of one eigenvector (overlap > 1/2) and which are distinct eigenvalues.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>

#include "batched.cuh"

namespace qmbed {

namespace {

constexpr int kMaxComp = 8;
constexpr int kMaxSectors = 128;
constexpr int kMaxCand = 8;          // Ritz candidates kept per pair (two per wanted eigenvalue)
constexpr int kRowsPerItem = 256;    // rows of one reduction item: 8 warps x 32 rows
constexpr int kThreads = 256;
constexpr int kChunkSteps = 10;      // Lanczos steps per persistent launch (one graph replay)
constexpr unsigned kSpinLimit = 1u << 22;  // barrier polls (with 64 ns sleeps: about a quarter second)

enum ScanStatus : int { kStatusRunning = 0, kStatusBarrierTimeout = 1 };

struct CompRows {
  const void* row_ptr;
  const uint32_t* cols;
  const double* vals;
  const double* diag;
  int row_ptr64;
  int diag_complex;
};

struct SectorDesc {
  uint64_t row0, n, item0, items;
  const uint16_t* weights;
  double* buf[3];            // Lanczos vectors (roles rotate with the step)
  double* ritz[kMaxCand];    // second pass: Ritz vector accumulators
  CompRows comp[kMaxComp];
};

// Device state shared by the persistent kernel, the check kernel and the host.
struct ScanState {
  unsigned barrier_count, barrier_gen;
  int status;                // ScanStatus
  int step;                  // steps completed in this pass
  int pass;                  // 1: search, 2: Ritz vectors
  int active;                // pairs not yet converged (pass 1)
  int target_steps;          // pass 2: steps to run (max over pairs of m_p)
  int pad;
};

struct ScanArgs {
  const SectorDesc* sec;
  int ns, P, K, cols, points, eigenpairs, max_steps, ncand;
  uint64_t total_rows, total_items;
  const double* coef;        // K x P
  double* partial;           // total_items x P
  double* alpha;             // max_steps x cols
  double* beta;              // (max_steps + 1) x cols; row max_steps: start-vector norms
  int* length;               // step at which beta vanished (Krylov space exhausted), -1 before
  int* stop;                 // pass-1 step count at convergence per pair (-1: running)
  double* cand_s;            // cols x ncand x max_steps: eigenvectors of T_m for the candidates
  double* cand_theta;        // cols x ncand
  double* top;               // cols: largest Ritz value at convergence
  int* sector_gate;          // rows of sector s take part in step j only while j < sector_gate[s]
  int* sector_running;       // pass 1: columns of sector s still running
  double tolerance;
  uint64_t seed;
  ScanState* state;
};

__device__ __forceinline__ int find_sector(const uint64_t* starts, int ns, uint64_t g) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (starts[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint64_t row_begin(const CompRows& c, uint64_t r) {
  return c.row_ptr64 ? static_cast<const uint64_t*>(c.row_ptr)[r] : static_cast<const uint32_t*>(c.row_ptr)[r];
}

// Grid-wide barrier with a bounded spin. Returns false when any block timed
// out (then every block leaves the kernel at its next barrier).
__device__ bool grid_sync(ScanState* st, unsigned blocks) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    volatile int* status = &st->status;
    if (*status != kStatusRunning) {
      ok = 0;
    } else {
      volatile unsigned* gen = &st->barrier_gen;
      const unsigned g = *gen;
      __threadfence();
      const unsigned arrived = atomicAdd(&st->barrier_count, 1u);
      if (arrived == blocks - 1) {
        st->barrier_count = 0;
        __threadfence();
        atomicAdd(&st->barrier_gen, 1u);
      } else {
        unsigned polls = 0;
        while (*gen == g) {
          if (++polls > kSpinLimit || *status != kStatusRunning) {
            atomicExch(&st->status, kStatusBarrierTimeout);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return ok != 0;
}

// The vector roles at step j: z_j (current), z_{j-1} (previous), work.
__device__ __forceinline__ void roles(int j, int& cur, int& prev, int& work) {
  cur = j % 3;
  prev = (j + 2) % 3;
  work = (j + 1) % 3;
}

// RPW rows per warp (1: a warp per row, 2: a half-warp per row with twice
// the points per lane) of all sectors: work = H(s, p) cur - beta_{j-1} prev,
// and in the second pass ritz_i += s_i[j] cur for the pairs still inside m_p.
template <int PPL, bool PASS2, int RPW>
__device__ void phase_apply(const ScanArgs& a, const uint64_t* starts, const double* c, int j) {
  constexpr int P = 32 * PPL;
  constexpr int LPR = 32 / RPW;   // lanes per row
  constexpr int PL = PPL * RPW;   // points per lane
  int cur, prev, work;
  roles(j, cur, prev, work);
  const int lane = threadIdx.x & 31;
  const int sl = lane % LPR;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t gw = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; gw * RPW < a.total_rows;
       gw += warps) {
    const uint64_t g = gw * RPW + static_cast<uint64_t>(lane / LPR);
    if (g >= a.total_rows) continue;
    const int s = find_sector(starts, a.ns, g);
    if (j >= a.sector_gate[s]) continue;  // every column of the sector is done
    const SectorDesc& d = a.sec[s];
    const uint64_t r = g - d.row0;
    const double* z = d.buf[cur];
    double are[PL], aim[PL], dsum[PL];
#pragma unroll
    for (int q = 0; q < PL; ++q) are[q] = aim[q] = dsum[q] = 0.0;
    for (int k = 0; k < a.K; ++k) {
      const CompRows& cr = d.comp[k];
      double ck[PL];
#pragma unroll
      for (int q = 0; q < PL; ++q) ck[q] = c[k * P + sl * PL + q];
      const uint64_t begin = row_begin(cr, r), end = row_begin(cr, r + 1);
      for (uint64_t e = begin; e < end; ++e) {
        const uint64_t col = cr.cols[e];
        const double vr = cr.vals[2 * e], vi = cr.vals[2 * e + 1];
        const double2* zc = reinterpret_cast<const double2*>(z) + col * P + sl * PL;
#pragma unroll
        for (int q = 0; q < PL; ++q) {
          const double2 x = zc[q];
          are[q] = fma(ck[q], vr * x.x - vi * x.y, are[q]);
          aim[q] = fma(ck[q], vr * x.y + vi * x.x, aim[q]);
        }
      }
      const double dr = cr.diag_complex ? cr.diag[2 * r] : cr.diag[r];
#pragma unroll
      for (int q = 0; q < PL; ++q) dsum[q] = fma(ck[q], dr, dsum[q]);
    }
    const double2* zs = reinterpret_cast<const double2*>(z) + r * P + sl * PL;
    const double2* pv = reinterpret_cast<const double2*>(d.buf[prev]) + r * P + sl * PL;
    double2* o = reinterpret_cast<double2*>(d.buf[work]) + r * P + sl * PL;
#pragma unroll
    for (int q = 0; q < PL; ++q) {
      const double2 x = zs[q];
      double wr = are[q] + dsum[q] * x.x, wi = aim[q] + dsum[q] * x.y;
      const int colidx = s * P + sl * PL + q;
      if (j > 0) {
        const double b = a.beta[static_cast<uint64_t>(j - 1) * a.cols + colidx];
        const double2 y = pv[q];
        wr -= b * y.x;
        wi -= b * y.y;
      }
      o[q] = make_double2(wr, wi);
      if (PASS2 && j < a.stop[colidx]) {
        for (int i = 0; i < a.ncand; ++i) {
          const double si = a.cand_s[(static_cast<uint64_t>(colidx) * a.ncand + i) * a.max_steps + j];
          double2* acc = reinterpret_cast<double2*>(d.ritz[i]) + r * P + sl * PL + q;
          double2 v = *acc;
          v.x = fma(si, x.x, v.x);
          v.y = fma(si, x.y, v.y);
          *acc = v;
        }
      }
    }
  }
}

// Reduction items (256 rows of one sector each). MODE 0: partial = sum_r R_r
// Re(conj(cur) work) (alpha); MODE 1: work -= alpha cur and partial =
// sum_r R_r |work|^2 (beta^2; alpha null for the start vector's norm).
template <int PPL, int MODE>
__device__ void phase_reduce(const ScanArgs& a, const uint64_t* item_starts, int ia, int ib, const double* alpha,
                             int j) {
  constexpr int P = 32 * PPL;
  __shared__ double red[kThreads / 32][P];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t item = blockIdx.x; item < a.total_items; item += gridDim.x) {
    const int s = find_sector(item_starts, a.ns, item);
    if (j >= a.sector_gate[s]) continue;  // block-uniform: one item per block iteration
    const SectorDesc& d = a.sec[s];
    const uint64_t local = item - d.item0;
    double acc[PPL];
#pragma unroll
    for (int q = 0; q < PPL; ++q) acc[q] = 0.0;
    double al[PPL];
#pragma unroll
    for (int q = 0; q < PPL; ++q) al[q] = (MODE == 1 && alpha) ? alpha[static_cast<uint64_t>(s) * P + lane * PPL + q] : 0.0;
    const uint64_t r0 = local * kRowsPerItem;
    for (int i = warp; i < kRowsPerItem; i += kThreads / 32) {
      const uint64_t r = r0 + i;
      if (r >= d.n) break;
      const double w = d.weights ? static_cast<double>(d.weights[r]) : 1.0;
      double2* x = reinterpret_cast<double2*>(d.buf[ia]) + r * P + lane * PPL;
      const double2* y = reinterpret_cast<const double2*>(d.buf[ib]) + r * P + lane * PPL;
#pragma unroll
      for (int q = 0; q < PPL; ++q) {
        double2 u = x[q];
        const double2 v = y[q];
        if (MODE == 0) {
          acc[q] = fma(w, u.x * v.x + u.y * v.y, acc[q]);
        } else {
          u.x -= al[q] * v.x;
          u.y -= al[q] * v.y;
          if (alpha) x[q] = u;
          acc[q] = fma(w, u.x * u.x + u.y * u.y, acc[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < PPL; ++q) red[warp][lane * PPL + q] = acc[q];
    __syncthreads();
    if (threadIdx.x < P) {
      double t = 0.0;
      for (int w8 = 0; w8 < kThreads / 32; ++w8) t += red[w8][threadIdx.x];
      a.partial[item * P + threadIdx.x] = t;
    }
    __syncthreads();
  }
}

// out[c] = sum over the sector's items of partial (in item order); SQRT: the
// square root, and the first step whose beta falls below 1e-12 (scale) is
// recorded as the exhausted Krylov length.
__device__ void phase_finish(const ScanArgs& a, double* out, bool sqrt_mode, int step, const double* alpha) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < static_cast<uint64_t>(a.cols);
       t += stride) {
    const int s = static_cast<int>(t / a.P), p = static_cast<int>(t % a.P);
    double v = 0.0;
    for (uint64_t b = a.sec[s].item0; b < a.sec[s].item0 + a.sec[s].items; ++b) v += a.partial[b * a.P + p];
    if (sqrt_mode) {
      v = sqrt(fmax(v, 0.0));
      const double scale = alpha ? fmax(fabs(alpha[t]), 1.0) : 1.0;
      if (step >= 0 && a.length[t] < 0 && v <= 1.0e-12 * scale) a.length[t] = step + 1;
    }
    out[t] = v;
  }
}

// dst = src / beta (0 where beta vanished), one warp per row.
template <int PPL>
__device__ void phase_scale(const ScanArgs& a, const uint64_t* starts, int isrc, int idst, const double* beta, int j) {
  constexpr int P = 32 * PPL;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < a.total_rows;
       g += warps) {
    const int s = find_sector(starts, a.ns, g);
    if (j >= a.sector_gate[s]) continue;
    const SectorDesc& d = a.sec[s];
    const uint64_t r = g - d.row0;
    const double2* x = reinterpret_cast<const double2*>(d.buf[isrc]) + r * P + lane * PPL;
    double2* o = reinterpret_cast<double2*>(d.buf[idst]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const double b = beta[static_cast<uint64_t>(s) * P + lane * PPL + q];
      const double inv = b > 1.0e-300 ? 1.0 / b : 0.0;
      const double2 v = x[q];
      o[q] = make_double2(v.x * inv, v.y * inv);
    }
  }
}

// Start vectors: real parts uniform in [-0.5, 0.5) from a SplitMix64 hash of
// (seed, sector, point, row), written to `idst`.
template <int PPL>
__device__ void phase_init(const ScanArgs& a, const uint64_t* starts, int idst) {
  constexpr int P = 32 * PPL;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < a.total_rows;
       g += warps) {
    const int s = find_sector(starts, a.ns, g);
    const SectorDesc& d = a.sec[s];
    const uint64_t r = g - d.row0;
    double2* o = reinterpret_cast<double2*>(d.buf[idst]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      uint64_t z = a.seed ^ (0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(s) * 4096 + lane * PPL + q + 1)) ^
                   (r * 0xd1b54a32d192ed03ULL);
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      z ^= z >> 31;
      o[q] = make_double2(static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0) - 0.5, 0.0);
    }
  }
}

// The persistent kernel: (when step == 0) the normalised start vectors, then
// up to kChunkSteps Lanczos steps of the current pass; the step counter in
// `state` advances once per completed step.
// MINB: the resident blocks per SM the register budget is compiled for (3:
// no spills; 4: 64 registers, more warps to hide the gathers' latency, a few
// spills); the autotuner picks between them.
// RPW: rows per warp in the apply phase (1 or 2), the other shape the
// autotuner chooses.
template <int PPL, bool PASS2, int MINB, int RPW>
__global__ void __launch_bounds__(kThreads, MINB) scan_chunk_kernel(const ScanArgs a) {
  constexpr int P = 32 * PPL;
  __shared__ double c[kMaxComp * P];
  __shared__ uint64_t starts[kMaxSectors], item_starts[kMaxSectors];
  for (int i = threadIdx.x; i < a.K * P; i += blockDim.x) c[i] = a.coef[i];
  for (int i = threadIdx.x; i < a.ns; i += blockDim.x) {
    starts[i] = a.sec[i].row0;
    item_starts[i] = a.sec[i].item0;
  }
  __syncthreads();
  const unsigned blocks = gridDim.x;
  ScanState* st = a.state;
  volatile int* vstep = &st->step;
  int j = *vstep;
  const int limit = PASS2 ? st->target_steps : a.max_steps;
  if (PASS2 ? j >= limit : (st->active == 0 || j >= limit)) return;
  double* beta0 = a.beta + static_cast<uint64_t>(a.max_steps) * a.cols;
  if (j == 0) {
    // z_0 = random / ||random||_R, built in the `work` role of step 0 then scaled into `cur`
    int cur, prev, work;
    roles(0, cur, prev, work);
    phase_init<PPL>(a, starts, work);
    if (!grid_sync(st, blocks)) return;
    phase_reduce<PPL, 1>(a, item_starts, work, work, nullptr, 0);
    if (!grid_sync(st, blocks)) return;
    phase_finish(a, beta0, true, -1, nullptr);
    if (!grid_sync(st, blocks)) return;
    phase_scale<PPL>(a, starts, work, cur, beta0, 0);
    if (!grid_sync(st, blocks)) return;
  }
  for (int n = 0; n < kChunkSteps && j < limit; ++n, ++j) {
    int cur, prev, work;
    roles(j, cur, prev, work);
    double* alpha_j = a.alpha + static_cast<uint64_t>(j) * a.cols;
    double* beta_j = a.beta + static_cast<uint64_t>(j) * a.cols;
    phase_apply<PPL, PASS2, RPW>(a, starts, c, j);
    if (!grid_sync(st, blocks)) return;
    phase_reduce<PPL, 0>(a, item_starts, cur, work, nullptr, j);
    if (!grid_sync(st, blocks)) return;
    phase_finish(a, alpha_j, false, j, nullptr);
    if (!grid_sync(st, blocks)) return;
    phase_reduce<PPL, 1>(a, item_starts, work, cur, alpha_j, j);
    if (!grid_sync(st, blocks)) return;
    phase_finish(a, beta_j, true, PASS2 ? -1 : j, alpha_j);
    if (!grid_sync(st, blocks)) return;
    // z_{j+1} = work / beta_j in place: step j+1 sees this buffer as `cur` and z_j as `prev`
    phase_scale<PPL>(a, starts, work, work, beta_j, j);
    if (!grid_sync(st, blocks)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) *vstep = j + 1;
  }
}

// ---------------------------------------------------------------------------
// Tridiagonal work per pair (one thread each)
// ---------------------------------------------------------------------------

struct Tri {
  const double* alpha;
  const double* beta;
  int cols, t, m;
  __device__ double a(int j) const { return alpha[static_cast<size_t>(j) * cols + t]; }
  __device__ double b(int j) const { return beta[static_cast<size_t>(j) * cols + t]; }
};

__device__ int count_below(const Tri& T, double x) {
  int c = 0;
  double q = T.a(0) - x;
  if (q < 0) ++c;
  for (int j = 1; j < T.m; ++j) {
    if (q == 0.0) q = 1e-300;
    const double bb = T.b(j - 1);
    q = T.a(j) - x - bb * bb / q;
    if (q < 0) ++c;
  }
  return c;
}

// i-th smallest eigenvalue of T by Sturm bisection (Gershgorin start).
__device__ double tri_eigenvalue(const Tri& T, int i, double lo, double hi) {
  double l = lo, h = hi;
  for (int it = 0; it < 200 && h - l > 2.0e-16 * fmax(fabs(l), fabs(h)) + 1e-300; ++it) {
    const double mid = 0.5 * (l + h);
    if (count_below(T, mid) > i) h = mid;
    else l = mid;
  }
  return 0.5 * (l + h);
}

// Eigenvector of T for the eigenvalue theta by two steps of inverse
// iteration (LU of T - theta' I without pivoting, theta' nudged off theta);
// written to s[0..m) with unit norm. Returns its last component.
__device__ double tri_vector(const Tri& T, double theta, double* s, double* work) {
  const int m = T.m;
  const double shift = theta + 1.0e-13 * fmax(fabs(theta), 1.0);
  for (int j = 0; j < m; ++j) s[j] = 1.0 / sqrt(static_cast<double>(m));
  for (int sweep = 0; sweep < 2; ++sweep) {
    // forward elimination: d_j = a_j - shift - b_{j-1}^2 / d_{j-1}; rhs likewise
    double d = T.a(0) - shift;
    if (d == 0.0) d = 1e-300;
    work[0] = d;
    double y = s[0];
    s[0] = y;
    for (int j = 1; j < m; ++j) {
      const double l = T.b(j - 1) / d;
      d = T.a(j) - shift - l * T.b(j - 1);
      if (d == 0.0) d = 1e-300;
      work[j] = d;
      s[j] = s[j] - l * s[j - 1];
    }
    // back substitution
    s[m - 1] /= work[m - 1];
    for (int j = m - 2; j >= 0; --j) s[j] = (s[j] - T.b(j) * s[j + 1]) / work[j];
    double norm = 0.0;
    for (int j = 0; j < m; ++j) norm += s[j] * s[j];
    norm = sqrt(norm);
    for (int j = 0; j < m; ++j) s[j] /= norm;
  }
  return s[m - 1];
}

// Pass-1 convergence check after `step` steps, for every pair still running.
// The Ritz values are grouped into clusters (values within 1e-8 max(|theta|,
// 1) of the cluster's first); copies of one eigenvalue from lost
// orthogonality form such clusters, and so would two genuinely close
// eigenvalues. A pair converges when the first member of each of its lowest
// `eigenpairs` clusters has a residual estimate |beta_m s_m| of at most
// 0.5 tol max(|theta|, 1). The candidates kept for the second pass are these
// first members and, where its estimate is as small, each cluster's second
// member; the second pass decides from the Ritz vectors whether a second
// member is a copy (overlap above 1/2) or a distinct eigenvalue. Also
// recorded: m and the top Ritz value. When the last column of a sector stops,
// the sector's rows leave the recurrence.
__global__ void scan_check_kernel(const ScanArgs a, double* work_all) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = a.state->step;
  if (t >= a.cols || a.stop[t] >= 0 || a.stop[t] <= -2 || step == 0) return;
  int m = step;
  const bool exhausted = a.length[t] > 0 && a.length[t] <= step;
  if (exhausted) m = a.length[t];
  const bool check = exhausted || step % kChunkSteps == 0 || step >= a.max_steps;
  if (!check) return;
  Tri T{a.alpha, a.beta, a.cols, t, m};
  double lo = 1e300, hi = -1e300;
  for (int j = 0; j < m; ++j) {
    const double off = (j > 0 ? fabs(T.b(j - 1)) : 0.0) + (j + 1 < m ? fabs(T.b(j)) : 0.0);
    lo = fmin(lo, T.a(j) - off);
    hi = fmax(hi, T.a(j) + off);
  }
  double* s = a.cand_s + static_cast<size_t>(t) * a.ncand * a.max_steps;
  double* work = work_all + static_cast<size_t>(t) * a.max_steps;
  const double beta_m = exhausted ? 0.0 : T.b(m - 1);
  int nc = 0, clusters = 0, members = 0;
  double cluster_value = 0.0;
  bool converged = true;
  for (int i = 0; i < m && nc < a.ncand; ++i) {
    const double theta = tri_eigenvalue(T, i, lo, hi);
    const double scale = fmax(fabs(theta), 1.0);
    if (clusters == 0 || theta - cluster_value > 1.0e-8 * scale) {
      if (clusters == a.eigenpairs) break;
      ++clusters;
      cluster_value = theta;
      members = 0;
    }
    if (members == 2) continue;
    ++members;
    double* v = s + static_cast<size_t>(nc) * a.max_steps;
    const bool small = fabs(beta_m * tri_vector(T, theta, v, work)) <= 0.5 * a.tolerance * scale;
    if (members == 1) {
      if (!small) converged = false;
    } else if (!small) {
      continue;  // a copy still forming: not a candidate
    }
    a.cand_theta[static_cast<size_t>(t) * a.ncand + nc] = theta;
    ++nc;
  }
  if (clusters < a.eigenpairs && m > nc) converged = false;
  if (!converged && !exhausted && step < a.max_steps) return;
  for (int i = nc; i < a.ncand; ++i) a.cand_theta[static_cast<size_t>(t) * a.ncand + i] = NAN;
  a.top[t] = tri_eigenvalue(T, m - 1, lo, hi);
  a.stop[t] = converged ? m : -2 - m;  // -2 - m: stopped at max_steps without convergence
  atomicSub(&a.state->active, 1);
  const int sector = t / a.P;
  if (atomicSub(&a.sector_running[sector], 1) == 1) a.sector_gate[sector] = step;  // the sector's last column
}

// Second-pass results: for candidate i of every pair, sums over the rows of
// R |v|^2, R Re(conj(v) H v), R |H v - theta v|^2 and the overlaps R Re(conj(v_i) v_k).
template <int PPL>
__global__ void __launch_bounds__(kThreads) scan_verify_kernel(const SectorDesc* __restrict__ sec, int ns, int P,
                                                               int ncand, int cand, const double* __restrict__ theta,
                                                               int hv_buf, double* __restrict__ partial) {
  // partial[item][c][q]: q = 0 |v|^2, 1 v.Hv, 2 |Hv - theta v|^2, 3 + k overlap with candidate k
  const int s_count = ns;
  __shared__ uint64_t item_starts[kMaxSectors];
  for (int i = threadIdx.x; i < s_count; i += blockDim.x) item_starts[i] = sec[i].item0;
  __syncthreads();
  const int s = find_sector(item_starts, s_count, blockIdx.x);
  const SectorDesc& d = sec[s];
  const uint64_t local = blockIdx.x - d.item0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int Q = 3 + kMaxCand;
  double acc[PPL][Q];
#pragma unroll
  for (int q = 0; q < PPL; ++q)
#pragma unroll
    for (int u = 0; u < Q; ++u) acc[q][u] = 0.0;
  const uint64_t r0 = local * kRowsPerItem;
  for (int i = warp; i < kRowsPerItem; i += kThreads / 32) {
    const uint64_t r = r0 + i;
    if (r >= d.n) break;
    const double w = d.weights ? static_cast<double>(d.weights[r]) : 1.0;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const uint64_t off = r * P + lane * PPL + q;
      const int colidx = s * P + lane * PPL + q;
      const double2 v = reinterpret_cast<const double2*>(d.ritz[cand])[off];
      const double2 h = reinterpret_cast<const double2*>(d.buf[hv_buf])[off];
      const double th = theta[static_cast<size_t>(colidx) * ncand + cand];
      const double rr = h.x - th * v.x, ri = h.y - th * v.y;
      acc[q][0] = fma(w, v.x * v.x + v.y * v.y, acc[q][0]);
      acc[q][1] = fma(w, v.x * h.x + v.y * h.y, acc[q][1]);
      acc[q][2] = fma(w, rr * rr + ri * ri, acc[q][2]);
      for (int k = 0; k < ncand; ++k) {
        const double2 u = reinterpret_cast<const double2*>(d.ritz[k])[off];
        acc[q][3 + k] = fma(w, v.x * u.x + v.y * u.y, acc[q][3 + k]);
      }
    }
  }
  __shared__ double red[kThreads / 32][64 * 2][1];
  for (int u = 0; u < Q; ++u) {
#pragma unroll
    for (int q = 0; q < PPL; ++q) red[warp][lane * PPL + q][0] = acc[q][u];
    __syncthreads();
    if (threadIdx.x < P) {
      double t = 0.0;
      for (int w8 = 0; w8 < kThreads / 32; ++w8) t += red[w8][threadIdx.x][0];
      partial[(static_cast<uint64_t>(blockIdx.x) * P + threadIdx.x) * Q + u] = t;
    }
    __syncthreads();
  }
}

// Applies H(s, p) to a Ritz accumulator (second-pass verification): one warp per row.
template <int PPL>
__global__ void __launch_bounds__(kThreads) scan_hv_kernel(const SectorDesc* __restrict__ sec, int ns, uint64_t total_rows,
                                                           int K, const double* __restrict__ coef, int cand, int out_buf) {
  constexpr int P = 32 * PPL;
  __shared__ double c[kMaxComp * P];
  __shared__ uint64_t starts[kMaxSectors];
  for (int i = threadIdx.x; i < K * P; i += blockDim.x) c[i] = coef[i];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) starts[i] = sec[i].row0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < total_rows; g += warps) {
    const int s = find_sector(starts, ns, g);
    const SectorDesc& d = sec[s];
    const uint64_t r = g - d.row0;
    const double* z = d.ritz[cand];
    double are[PPL], aim[PPL], dsum[PPL];
#pragma unroll
    for (int q = 0; q < PPL; ++q) are[q] = aim[q] = dsum[q] = 0.0;
    for (int k = 0; k < K; ++k) {
      const CompRows& cr = d.comp[k];
      double ck[PPL];
#pragma unroll
      for (int q = 0; q < PPL; ++q) ck[q] = c[k * P + lane * PPL + q];
      const uint64_t begin = row_begin(cr, r), end = row_begin(cr, r + 1);
      for (uint64_t e = begin; e < end; ++e) {
        const uint64_t col = cr.cols[e];
        const double vr = cr.vals[2 * e], vi = cr.vals[2 * e + 1];
        const double2* zc = reinterpret_cast<const double2*>(z) + col * P + lane * PPL;
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
          const double2 x = zc[q];
          are[q] = fma(ck[q], vr * x.x - vi * x.y, are[q]);
          aim[q] = fma(ck[q], vr * x.y + vi * x.x, aim[q]);
        }
      }
      const double dr = cr.diag_complex ? cr.diag[2 * r] : cr.diag[r];
#pragma unroll
      for (int q = 0; q < PPL; ++q) dsum[q] = fma(ck[q], dr, dsum[q]);
    }
    const double2* zs = reinterpret_cast<const double2*>(z) + r * P + lane * PPL;
    double2* o = reinterpret_cast<double2*>(d.buf[out_buf]) + r * P + lane * PPL;
#pragma unroll
    for (int q = 0; q < PPL; ++q) {
      const double2 x = zs[q];
      o[q] = make_double2(are[q] + dsum[q] * x.x, aim[q] + dsum[q] * x.y);
    }
  }
}

// A kernel that waits at the grid barrier for one more block than it has:
// the bounded spin must end with kStatusBarrierTimeout (used by the test of
// the time-out path).
__global__ void barrier_selftest_kernel(ScanState* st) { grid_sync(st, gridDim.x + 1); }

template <typename F>
void by_points(int P, F&& f) {
  if (P == 32) f(std::integral_constant<int, 1>{});
  else f(std::integral_constant<int, 2>{});
}

}  // namespace

int scan_barrier_selftest(int device) {
  QMBED_CUDA(cudaSetDevice(device));
  DeviceBuffer state(sizeof(ScanState));
  QMBED_CUDA(cudaMemset(state.get(), 0, sizeof(ScanState)));
  int sms = 148, per_sm = 0;
  QMBED_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  QMBED_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, barrier_selftest_kernel, 32, 0));
  ScanState* st = state.as<ScanState>();
  void* args[] = {&st};
  const unsigned grid = static_cast<unsigned>(std::max(1, std::min(2, per_sm)) * sms);
  QMBED_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(barrier_selftest_kernel), dim3(grid), dim3(32), args,
                                         0, nullptr));
  QMBED_LAUNCH_CHECK();
  QMBED_CUDA(cudaDeviceSynchronize());
  ScanState host{};
  QMBED_CUDA(cudaMemcpy(&host, state.get(), sizeof(ScanState), cudaMemcpyDeviceToHost));
  return host.status;
}

ScanResult scan_lowest(const std::vector<std::vector<const SpinOperator*>>& components,
                       const std::vector<double>& coefficients, int points, int eigenpairs, double tolerance,
                       int max_steps, uint64_t seed, BlockOps& ops) {
  const int ns = static_cast<int>(components.size());
  if (ns < 1 || ns > kMaxSectors) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 128 sectors");
  const int K = static_cast<int>(components[0].size());
  if (K < 1 || K > kMaxComp) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 8 components");
  if (points < 1 || points > 64) raise(QMBED_INVALID_OPTIONS, "a scan takes 1 to 64 points");
  if (eigenpairs < 1 || eigenpairs > 4) raise(QMBED_INVALID_OPTIONS, "a scan returns 1 to 4 eigenvalues per pair");
  if (!(tolerance > 0.0) || max_steps < 1) raise(QMBED_INVALID_OPTIONS, "tolerance and steps must be positive");
  if (static_cast<int>(coefficients.size()) != points * K) raise(QMBED_DIMENSION_MISMATCH, "coefficients must be points x components");
  const auto t_start = std::chrono::steady_clock::now();
  const int P = points <= 32 ? 32 : 64;
  const int ncand = 2 * eigenpairs;
  const cudaStream_t stream = ops.stream();
  int device = 0;
  QMBED_CUDA(cudaGetDevice(&device));
  // coefficients padded to P columns by repeating the last point
  std::vector<double> coef(static_cast<size_t>(K) * P);
  for (int k = 0; k < K; ++k)
    for (int p = 0; p < P; ++p) coef[static_cast<size_t>(k) * P + p] = coefficients[static_cast<size_t>(std::min(p, points - 1)) * K + k];
  std::vector<SectorDesc> desc(ns);
  uint64_t rows = 0, items = 0;
  size_t set_bytes = 0;  // one vector set (every sector's rows x P complex FP64)
  for (int s = 0; s < ns; ++s) {
    if (static_cast<int>(components[s].size()) != K) raise(QMBED_DIMENSION_MISMATCH, "every sector needs the same components");
    const SpinOperator* first = components[s][0];
    SectorDesc& d = desc[s];
    std::memset(&d, 0, sizeof(d));
    d.n = first->dim();
    d.row0 = rows;
    d.item0 = items;
    d.items = (d.n + kRowsPerItem - 1) / kRowsPerItem;
    d.weights = first->basis().symmetric() ? first->basis().orbits() : nullptr;
    rows += d.n;
    items += d.items;
    set_bytes += d.n * P * 16;
    for (int k = 0; k < K; ++k) {
      const SpinOperator* op = components[s][k];
      if (op->dim() != d.n || &op->basis() != &first->basis())
        raise(QMBED_DIMENSION_MISMATCH, "the components of a sector must share its basis");
      const SpinOperator::ExplicitRows er = op->explicit_rows();
      d.comp[k] = CompRows{er.row_ptr, er.cols, er.values, er.diag, er.row_ptr64 ? 1 : 0, er.diag_complex ? 1 : 0};
    }
  }
  const int cols = ns * P;
  DeviceBuffer lanczos_mem(3 * set_bytes), ritz_mem(static_cast<size_t>(ncand) * set_bytes);
  DeviceBuffer desc_dev(ns * sizeof(SectorDesc)), coef_dev(coef.size() * sizeof(double));
  constexpr int Q = 3 + kMaxCand;
  DeviceBuffer partial(std::max<uint64_t>(items, 1) * P * Q * sizeof(double));
  DeviceBuffer alpha_hist(static_cast<size_t>(max_steps) * cols * sizeof(double));
  DeviceBuffer beta_hist(static_cast<size_t>(max_steps + 1) * cols * sizeof(double));
  DeviceBuffer length(cols * sizeof(int)), stop(cols * sizeof(int));
  DeviceBuffer cand_s(static_cast<size_t>(cols) * ncand * max_steps * sizeof(double));
  DeviceBuffer cand_theta(static_cast<size_t>(cols) * ncand * sizeof(double)), top(cols * sizeof(double));
  DeviceBuffer tri_work(static_cast<size_t>(cols) * max_steps * sizeof(double));
  DeviceBuffer state(sizeof(ScanState));
  DeviceBuffer gate(ns * sizeof(int)), running(ns * sizeof(int));
  size_t offset = 0, roffset = 0;
  for (int s = 0; s < ns; ++s) {
    for (int b = 0; b < 3; ++b) {
      desc[s].buf[b] = reinterpret_cast<double*>(lanczos_mem.as<char>() + offset);
      offset += desc[s].n * P * 16;
    }
    for (int i = 0; i < ncand; ++i) {
      desc[s].ritz[i] = reinterpret_cast<double*>(ritz_mem.as<char>() + roffset);
      roffset += desc[s].n * P * 16;
    }
  }
  QMBED_CUDA(cudaMemcpyAsync(desc_dev.get(), desc.data(), ns * sizeof(SectorDesc), cudaMemcpyHostToDevice, stream));
  QMBED_CUDA(cudaMemcpyAsync(coef_dev.get(), coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  QMBED_CUDA(cudaMemsetAsync(length.get(), 0xff, cols * sizeof(int), stream));  // -1: not exhausted
  QMBED_CUDA(cudaMemsetAsync(stop.get(), 0xff, cols * sizeof(int), stream));    // -1: running
  QMBED_CUDA(cudaMemsetAsync(ritz_mem.get(), 0, static_cast<size_t>(ncand) * set_bytes, stream));
  {
    const std::vector<int> gates(ns, max_steps), counts(ns, P);
    QMBED_CUDA(cudaMemcpyAsync(gate.get(), gates.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
    QMBED_CUDA(cudaMemcpyAsync(running.get(), counts.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
  }
  ScanState init{};
  init.pass = 1;
  init.active = cols;
  QMBED_CUDA(cudaMemcpyAsync(state.get(), &init, sizeof(ScanState), cudaMemcpyHostToDevice, stream));

  ScanArgs a{};
  a.sec = desc_dev.as<SectorDesc>();
  a.ns = ns;
  a.P = P;
  a.K = K;
  a.cols = cols;
  a.points = points;
  a.eigenpairs = eigenpairs;
  a.max_steps = max_steps;
  a.ncand = ncand;
  a.total_rows = rows;
  a.total_items = items;
  a.coef = coef_dev.as<double>();
  a.partial = partial.as<double>();
  a.alpha = alpha_hist.as<double>();
  a.beta = beta_hist.as<double>();
  a.length = length.as<int>();
  a.stop = stop.as<int>();
  a.cand_s = cand_s.as<double>();
  a.cand_theta = cand_theta.as<double>();
  a.top = top.as<double>();
  a.sector_gate = gate.as<int>();
  a.sector_running = running.as<int>();
  a.tolerance = tolerance;
  a.seed = seed;
  a.state = state.as<ScanState>();

  ScanResult result;
  ScanState* host_state = nullptr;
  QMBED_CUDA(cudaMallocHost(&host_state, sizeof(ScanState)));
  *host_state = ScanState{};
  host_state->active = 1;  // until the first chunk's copy arrives
  struct PinnedFree {
    ScanState* p;
    ~PinnedFree() { cudaFreeHost(p); }
  } pinned_guard{host_state};
  auto read_state = [&] {
    QMBED_CUDA(cudaMemcpyAsync(host_state, state.get(), sizeof(ScanState), cudaMemcpyDeviceToHost, stream));
    QMBED_CUDA(cudaStreamSynchronize(stream));
    if (host_state->status == kStatusBarrierTimeout)
      raise(QMBED_DEVICE_TIMEOUT, "batched scan: a grid barrier timed out (not every block of the persistent "
                                  "launch was resident)");
  };

  by_points(P, [&](auto ptag) {
    constexpr int PPL = decltype(ptag)::value;
    auto grid_of = [&](const void* kernel) {
      int per_sm = 0;
      QMBED_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
      if (per_sm < 1) raise(QMBED_UNSUPPORTED_BACKEND, "the persistent scan kernel does not fit on an SM");
      return static_cast<unsigned>(per_sm * ops.sms());
    };
    const void* k1 = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, false, 3, 1>);
    const void* k2 = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, true, 3, 1>);
    const void* k1_wide = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, false, 4, 1>);
    const void* k2_wide = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, true, 4, 1>);
    const void* k1_pair = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, false, 3, 2>);
    const void* k2_pair = reinterpret_cast<const void*>(scan_chunk_kernel<PPL, true, 3, 2>);
    unsigned grid1 = grid_of(k1), grid2 = grid_of(k2);
    const int max_per_sm1 = static_cast<int>(grid1 / ops.sms());
    const int wide_per_sm1 = static_cast<int>(grid_of(k1_wide) / ops.sms());
    const int wide_per_sm2 = static_cast<int>(grid_of(k2_wide) / ops.sms());
    const int check_grid = (cols + 127) / 128;
    double* tri = tri_work.as<double>();
    ScanArgs args = a;
    void* kargs[] = {&args};
    auto chunk = [&](bool pass2) {
      QMBED_CUDA(cudaLaunchCooperativeKernel(pass2 ? k2 : k1, dim3(pass2 ? grid2 : grid1), dim3(kThreads), kargs, 0,
                                             stream));
      QMBED_LAUNCH_CHECK();
      if (!pass2) {
        scan_check_kernel<<<check_grid, 128, 0, stream>>>(args, tri);
        QMBED_LAUNCH_CHECK();
      }
      QMBED_CUDA(cudaMemcpyAsync(host_state, state.get(), sizeof(ScanState), cudaMemcpyDeviceToHost, stream));
    };
    // Autotuner: the persistent launch's resident blocks per SM. More blocks
    // hide more gather latency, fewer make every grid barrier cheaper; the
    // first chunks of pass 1 (real work, all pairs active) run once per
    // candidate under CUDA events and the fastest shape is captured below
    // and kept for pass 2.
    result.tuned_blocks_per_sm = max_per_sm1;
    if (max_per_sm1 > 1 && rows >= (1ull << 16) && max_steps >= 6 * kChunkSteps) {
      // candidates: (register budget, rows per warp, blocks per SM)
      struct Shape {
        bool wide;
        int rpw;
        int per_sm;
      };
      const int pair_per_sm1 = static_cast<int>(grid_of(k1_pair) / ops.sms());
      std::vector<Shape> shapes{{false, 1, max_per_sm1}, {false, 2, pair_per_sm1}};
      if (wide_per_sm1 > max_per_sm1) shapes.push_back({true, 1, wide_per_sm1});
      if (max_per_sm1 > 1) shapes.push_back({false, 1, max_per_sm1 - 1});
      cudaEvent_t e0, e1;
      QMBED_CUDA(cudaEventCreate(&e0));
      QMBED_CUDA(cudaEventCreate(&e1));
      double best = std::numeric_limits<double>::infinity();
      Shape chosen = shapes.front();
      const void* k1_plain = k1;
      for (const Shape& shape : shapes) {
        k1 = shape.wide ? k1_wide : (shape.rpw == 2 ? k1_pair : k1_plain);
        grid1 = static_cast<unsigned>(shape.per_sm * ops.sms());
        QMBED_CUDA(cudaEventRecord(e0, stream));
        chunk(false);
        QMBED_CUDA(cudaEventRecord(e1, stream));
        QMBED_CUDA(cudaStreamSynchronize(stream));
        float ms = 0.0f;
        QMBED_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        result.tuning_ms.push_back(ms);
        if (ms < best) {
          best = ms;
          chosen = shape;
          result.tuned_blocks_per_sm = shape.per_sm;
          result.tuned_rows_per_warp = shape.rpw;
        }
        if (host_state->status == kStatusBarrierTimeout || host_state->active == 0 || host_state->step >= max_steps)
          break;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      k1 = chosen.wide ? k1_wide : (chosen.rpw == 2 ? k1_pair : k1_plain);
      k2 = chosen.wide ? k2_wide : (chosen.rpw == 2 ? k2_pair : k2);
      const int per_sm2 = chosen.wide ? wide_per_sm2
                                      : static_cast<int>(grid_of(chosen.rpw == 2 ? k2_pair : k2) / ops.sms());
      grid1 = static_cast<unsigned>(chosen.per_sm * ops.sms());
      grid2 = static_cast<unsigned>(std::min(chosen.per_sm, per_sm2) * ops.sms());
    }
    // Pass 1: one chunk captured in a graph, replayed until every pair stopped.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_ok = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (graph_ok) {
      chunk(false);
      graph_ok = cudaStreamEndCapture(stream, &graph) == cudaSuccess && graph &&
                 cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    }
    if (!graph_ok) {
      (void)cudaGetLastError();  // capture not available: launch the chunks directly
      cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(stream, &capture) == cudaSuccess && capture != cudaStreamCaptureStatusNone) {
        cudaGraph_t discarded = nullptr;
        cudaStreamEndCapture(stream, &discarded);
        if (discarded) cudaGraphDestroy(discarded);
      }
      if (graph) cudaGraphDestroy(graph);
      graph = nullptr;
      exec = nullptr;
    }
    result.graph = graph_ok;
    const int max_chunks = (max_steps + kChunkSteps - 1) / kChunkSteps + 1;
    for (int c = 0; c < max_chunks; ++c) {
      if (host_state->status == kStatusBarrierTimeout || host_state->active == 0 ||
          host_state->step >= max_steps)
        break;  // the tuning chunks may already have finished
      if (exec) QMBED_CUDA(cudaGraphLaunch(exec, stream));
      else chunk(false);
      QMBED_CUDA(cudaStreamSynchronize(stream));
      if (host_state->status == kStatusBarrierTimeout) break;
      if (host_state->active == 0 || host_state->step >= max_steps) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    read_state();
    result.total_steps = host_state->step;
    result.pass1_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();

    std::vector<int> host_stop(cols);
    QMBED_CUDA(cudaMemcpy(host_stop.data(), stop.get(), cols * sizeof(int), cudaMemcpyDeviceToHost));
    int target = 0;
    for (int c = 0; c < cols; ++c) {
      const int m = host_stop[c] >= 0 ? host_stop[c] : (host_stop[c] <= -2 ? -2 - host_stop[c] : 0);
      target = std::max(target, m);
      if ((c % P) < points) result.applications += static_cast<size_t>(m);
    }
    // Pass 2: the same recurrence from the same start vectors, accumulating
    // the candidates' Ritz vectors (the stop array now bounds each pair's steps).
    std::vector<int> bounded(cols);
    for (int c = 0; c < cols; ++c) bounded[c] = host_stop[c] >= 0 ? host_stop[c] : (host_stop[c] <= -2 ? -2 - host_stop[c] : 0);
    QMBED_CUDA(cudaMemcpyAsync(stop.get(), bounded.data(), cols * sizeof(int), cudaMemcpyHostToDevice, stream));
    // pass 2: a sector's rows take part while any of its columns needs the step
    std::vector<int> gates(ns, 0);
    for (int c = 0; c < cols; ++c) gates[c / P] = std::max(gates[c / P], bounded[c]);
    QMBED_CUDA(cudaMemcpyAsync(gate.get(), gates.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
    ScanState second{};
    second.pass = 2;
    second.target_steps = target;
    QMBED_CUDA(cudaMemcpyAsync(state.get(), &second, sizeof(ScanState), cudaMemcpyHostToDevice, stream));
    for (int c = 0; c * kChunkSteps < target + kChunkSteps; ++c) {
      chunk(true);
      QMBED_CUDA(cudaStreamSynchronize(stream));
      if (host_state->status == kStatusBarrierTimeout || host_state->step >= target) break;
    }
    read_state();
    result.pass2_steps = target;
    // Verification: H v for every candidate, then the per-pair sums.
    const int row_grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((rows * 32 + 255) / 256, 16ull * ops.sms())));
    std::vector<double> sums(static_cast<size_t>(cols) * ncand * Q, 0.0), host_partial;
    for (int i = 0; i < ncand; ++i) {
      scan_hv_kernel<PPL><<<row_grid, kThreads, 0, stream>>>(a.sec, ns, rows, K, a.coef, i, 0);
      QMBED_LAUNCH_CHECK();
      scan_verify_kernel<PPL><<<static_cast<unsigned>(items), kThreads, 0, stream>>>(a.sec, ns, P, ncand, i,
                                                                                     a.cand_theta, 0, a.partial);
      QMBED_LAUNCH_CHECK();
      host_partial.resize(static_cast<size_t>(items) * P * Q);
      QMBED_CUDA(cudaMemcpyAsync(host_partial.data(), a.partial, host_partial.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, stream));
      QMBED_CUDA(cudaStreamSynchronize(stream));
      for (int s = 0; s < ns; ++s)
        for (uint64_t b = desc[s].item0; b < desc[s].item0 + desc[s].items; ++b)
          for (int p = 0; p < P; ++p)
            for (int u = 0; u < Q; ++u)
              sums[((static_cast<size_t>(s) * P + p) * ncand + i) * Q + u] += host_partial[(b * P + p) * Q + u];
    }
    result.applications_verification = static_cast<size_t>(target) * points * ns + static_cast<size_t>(ncand) * points * ns;
    std::vector<double> theta(static_cast<size_t>(cols) * ncand), host_top(cols);
    QMBED_CUDA(cudaMemcpy(theta.data(), cand_theta.get(), theta.size() * sizeof(double), cudaMemcpyDeviceToHost));
    QMBED_CUDA(cudaMemcpy(host_top.data(), top.get(), cols * sizeof(double), cudaMemcpyDeviceToHost));
    result.eigenvalues.assign(static_cast<size_t>(ns) * points * eigenpairs, std::nan(""));
    result.residuals.assign(static_cast<size_t>(ns) * points * eigenpairs, std::nan(""));
    result.e_max.assign(static_cast<size_t>(ns) * points, std::nan(""));
    result.steps.assign(static_cast<size_t>(ns) * points, -1);
    bool all_ok = true;
    for (int s = 0; s < ns; ++s)
      for (int p = 0; p < points; ++p) {
        const int c = s * P + p;
        const size_t out = static_cast<size_t>(s) * points + p;
        result.steps[out] = host_stop[c] >= 0 ? host_stop[c] : -1;
        result.e_max[out] = host_top[c];
        auto S = [&](int i, int u) { return sums[(static_cast<size_t>(c) * ncand + i) * Q + u]; };
        // accept candidates in ascending order; a close candidate whose vector
        // overlaps an accepted one by more than 1/2 is a copy of it
        std::vector<int> accepted;
        for (int i = 0; i < ncand && static_cast<int>(accepted.size()) < eigenpairs; ++i) {
          const double th = theta[static_cast<size_t>(c) * ncand + i];
          if (std::isnan(th) || !(S(i, 0) > 0.0)) continue;
          bool copy = false;
          for (int k : accepted) {
            const double overlap = std::fabs(S(i, 3 + k)) / std::sqrt(S(i, 0) * S(k, 0));
            const double thk = theta[static_cast<size_t>(c) * ncand + k];
            if (std::fabs(th - thk) <= 1.0e-8 * std::max(std::fabs(th), 1.0) && overlap > 0.5) copy = true;
          }
          if (copy) {
            ++result.merged_copies;
            continue;
          }
          accepted.push_back(i);
        }
        for (size_t q = 0; q < accepted.size(); ++q) {
          const int i = accepted[q];
          const double th = theta[static_cast<size_t>(c) * ncand + i];
          const double res = std::sqrt(std::max(S(i, 2), 0.0) / S(i, 0));
          result.eigenvalues[out * eigenpairs + q] = th;
          result.residuals[out * eigenpairs + q] = res;
          const double rel = res / std::max(std::fabs(th), 1.0);
          result.max_relative_residual = std::max(result.max_relative_residual, rel);
          if (!(rel <= tolerance)) all_ok = false;
        }
        if (static_cast<int>(accepted.size()) < eigenpairs || host_stop[c] < 0) {
          all_ok = false;
          ++result.failed_pairs;
        }
      }
    result.verified = all_ok;
  });
  result.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  if (!result.verified)
    raise(QMBED_NON_CONVERGENCE, "solver did not converge after " + std::to_string(result.total_steps) +
                                     " iterations; " + std::to_string(result.failed_pairs) +
                                     " scan pairs without verified eigenpairs, largest relative residual " +
                                     std::to_string(result.max_relative_residual));
  return result;
}

}  // namespace qmbed
