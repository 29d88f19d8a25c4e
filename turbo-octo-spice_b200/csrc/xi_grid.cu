// xi_grid.cu — grid-sweep kernel of the XiEstimator pair count (Cartesian
// and observing coordinates) for catalogues whose first-axis coordinate takes
// few distinct values: forests on a common log-wavelength grid, whose
// distances are one function of loglam (h5healxi.cc:196-203).
//
// With U the sorted distinct first-axis values of the catalogue and a
// sightline contiguous on U (its pixel p has value U[f + p]), the run
// boundaries of xi_sweep.cuh for a row x1 = U[g] along any column sightline j
// are the entries of one table row, in column order:
//   B[g][t] - f_j clamped to [0, n_j],  t = 0 .. 2 n0 + 1,
// where B[g][t] is the first grid index g2 whose value passes the boundary
// predicate of a threshold T[k] against U[g] (side 1 for t <= n0, side 0
// after it; k_grid_table, engine.cu).  The row's columns are then the
// consecutive runs [B[t], B[t+1]), t = 0 .. 2 n0, each of one first-axis bin
// (run n0 is the |x1 - x2| < T[0] gap), so neighbouring lanes share a
// boundary: a lane reads one table entry per row and evaluates one column.
#include <algorithm>

#include "xi_sweep.cuh"

namespace tos {
namespace {

constexpr int kGridWarps = 4;  // warps per CTA of the grid-sweep kernel

// Runs of an item per pass: a pass holds m + 1 <= 32 consecutive boundaries
// of a row, so it owns m runs.
constexpr int kPassRuns = 31;
constexpr int kGridThreads = kGridWarps * 32;

// A grid-sweep lane's FP64 sums (7 XiBin sums and the pair count) of its run
// for two r_perp codes: the current code C in registers and C - 1 in shared
// memory.  Along the rows of an item a run's code grows slowly; the rows
// where the run straddles a code edge add to both.  A code leaves for the
// per-cell sums once, when the codes move past it; a code below C - 1 (rare)
// goes straight out.  Same adds per (item, bin) as RunAcc.
struct GridAcc {
  int C;             // code of the register sums (-1: nothing added yet)
  bool prev_used;    // the shared sums of code C - 1 hold something
  double s[8];
  double* prev;      // this lane's shared sums of code C - 1, field f at prev[f * kGridThreads]

  template <int COORD>
  __device__ __forceinline__ void flush_prev(const PairArgs& A, Dest d, int k) {
    if (!prev_used) return;
    double v[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) v[f] = prev[f * kGridThreads];
    acc_flush8<COORD>(A, d, k, C - 1, v);
    prev_used = false;
  }

  template <int COORD>
  __device__ __forceinline__ void add(const PairArgs& A, Dest d, int k, int cc, const double (&v)[8]) {
    if (C < 0) C = cc;
    if (cc == C) {
#pragma unroll
      for (int f = 0; f < 8; ++f) s[f] += v[f];
    } else if (cc == C - 1) {
#pragma unroll
      for (int f = 0; f < 8; ++f) prev[f * kGridThreads] = (prev_used ? prev[f * kGridThreads] : 0.0) + v[f];
      prev_used = true;
    } else if (cc == C + 1) {
      flush_prev<COORD>(A, d, k);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        prev[f * kGridThreads] = s[f];
        s[f] = v[f];
      }
      prev_used = true;
      C = cc;
    } else if (cc > C + 1) {
      flush_prev<COORD>(A, d, k);
      acc_flush8<COORD>(A, d, k, C, s);
#pragma unroll
      for (int f = 0; f < 8; ++f) s[f] = v[f];
      C = cc;
    } else {
      acc_flush8<COORD>(A, d, k, cc, v);  // below both codes: straight out
    }
  }

  template <int COORD>
  __device__ __forceinline__ void finish(const PairArgs& A, Dest d, int k) {
    flush_prev<COORD>(A, d, k);
    if (C >= 0) acc_flush8<COORD>(A, d, k, C, s);
  }
};

// One pass over the rows of an item: runs t0 .. t0 + m - 1 of every row,
// run t = [B[t], B[t+1]) of the row's boundary table (k_grid_table, engine.cu)
// with the columns clamped to sightline j.  Boundary b (0 <= b <= m) of the
// pass sits on lane b + (m + 1) q of phase q = 0 .. P - 1, P = 32 / (m + 1);
// phase q takes rows g_lo + q, g_lo + q + P, ...  A lane evaluates its own
// boundary only: the column, its r_perp code and sightline j's prefix sums
// there.  The lane of boundary b owns run t0 + b and reads the run's far end
// from lane b + 1: when the two codes agree, every column of the run has that
// code (the code is non-decreasing along a row), so the run is added from the
// two prefix sums without evaluating anything else.  When they differ by one
// code (the common case: a run spans a few columns) the run has one change
// point, found by bisection between its first column and the neighbour's;
// otherwise the run's last column is evaluated and the run split by
// bisection.  Each lane sums its run into FP64
// registers across the rows (its first-axis bin is fixed; its r_perp code
// moves slowly from row to row) and adds them to the per-cell sums when its
// codes move on.
template <int COORD, bool MINPOS>
__device__ __forceinline__ void grid_pass(const PairArgs& A, const SweepItem& it, int fi, int fj, int t0,
                                          int m, int lane, double* prev, unsigned long long* stats) {
  const int n0 = (int)A.g.n0;
  const int nbd = 2 * n0 + 2;  // boundaries per table row
  const int P = 32 / (m + 1);
  const bool act = lane < (m + 1) * P;
  const int bi = act ? lane % (m + 1) : m;
  const int phase = act ? lane / (m + 1) : 0;
  const int t = t0 + bi;
  const bool owner = act && bi < m && t != n0;  // run n0 is the |x1 - x2| < T[0] gap
  const int k = (t < n0) ? n0 - 1 - t : t - n0 - 1;
  // the item in registers: the loop's flushes would force reloads from memory
  const int nj = it.nj, r_lo = it.r_lo, r_hi = it.r_hi;
  const Dest d = it.d;
  const double c = it.c;
  const float ap = it.ap, inv1sqf = A.inv1sqf;
  const float *rowl = it.rowl, *colx = it.colx;
  const PixPack* rowp = it.rowp;
  const double4* pre = it.pre;
  const uint16_t* tab = A.gq + (size_t)fi * nbd;  // row r: tab[r * nbd + t]
  // Rows where a run of the pass is non-empty: B[t0 + m] > fj and
  // B[t0] < fj + nj.  Table entries are non-decreasing along the rows, so
  // these rows form one interval (found the same way by every lane).
  int g_lo = r_lo, g_hi = r_hi;
  {
    int b = r_hi;
    while (g_lo < b) {
      const int mid = (g_lo + b) >> 1;
      if ((int)tab[(size_t)mid * nbd + t0 + m] > fj) b = mid; else g_lo = mid + 1;
    }
    int a = g_lo;
    while (a < g_hi) {
      const int mid = (a + g_hi) >> 1;
      if ((int)tab[(size_t)mid * nbd + t0] >= fj + nj) g_hi = mid; else a = mid + 1;
    }
  }
  if (g_hi <= g_lo) return;  // warp-uniform: every run of the pass is empty
  GridAcc acc;
  acc.C = -1;
  acc.prev_used = false;
  acc.prev = prev;
#pragma unroll
  for (int f = 0; f < 8; ++f) acc.s[f] = 0.0;
  unsigned rech = 0;
  unsigned long long n_eval = 0;
  const int n1 = (int)A.g.n1;
  const int iters = (g_hi - g_lo + P - 1) / P;  // the same for every phase (shuffles below)
  const uint16_t* tcol = tab + t;
  auto bound = [&](int row) { return min(max((int)tcol[(size_t)row * nbd] - fj, 0), nj); };
  // Software pipeline: the boundary of the row after next, and the column
  // value and prefix sums at the next row's boundary, load while this row is
  // evaluated (the column data depends on a boundary that is itself a load).
  int r = g_lo + phase;
  const int r0 = min(r, g_hi - 1), r1 = min(r + P, g_hi - 1);
  int b = bound(r0), nb = bound(r1);
  float x2 = colx[min(b, nj - 1)];
  double2 pwd = *reinterpret_cast<const double2*>(&pre[b]);
  double pl = pre[b].z;
  RowRaw cR = row_raw_packed(rowp, rowl, r0);
#pragma unroll 1
  for (int q = 0; q < iters; ++q, r += P) {
    const bool valid = act && r < g_hi;
    // loads for the rows ahead (the row values, broadcast loads that hit in
    // L1, one row ahead only)
    const float nx2 = colx[min(nb, nj - 1)];
    const double2 npwd = *reinterpret_cast<const double2*>(&pre[nb]);
    const double npl = pre[nb].z;
    const int r2 = min(r + 2 * P, g_hi - 1);
    const int nnb = bound(r2);
    const RowRaw nR = row_raw_packed(rowp, rowl, min(r + P, g_hi - 1));
    const RowV R = row_derive<COORD>(cR, ap, inv1sqf);
    // this lane's boundary: r_perp code of column b (of the last column when
    // b = nj: then it is the code of the last column of the run ending here)
    int code = 0;
    if (COORD == kCart && valid) code = perp_code<MINPOS>(A, R, x2, c, rech);
    const int be = __shfl_down_sync(kFull, b, 1);
    const int ce = __shfl_down_sync(kFull, code, 1);
    const double ewd = __shfl_down_sync(kFull, pwd.x, 1);
    const double ew = __shfl_down_sync(kFull, pwd.y, 1);
    const double el = __shfl_down_sync(kFull, pl, 1);
    if (valid && owner && be > b) {
      n_eval += (unsigned long long)(be - b);
      if (COORD == kObs) {
        add_sums<COORD>(A, d, R, k, 0, be - b, ewd - pwd.x, ew - pwd.y, el - pl, acc);
      } else if (code == ce) {
        if (code >= 0 && code < n1) add_sums<COORD>(A, d, R, k, code, be - b, ewd - pwd.x, ew - pwd.y, el - pl, acc);
      } else if (ce == code + 1) {
        // One code step between the run's first column and column hi (be,
        // or the last column nj - 1 when be = nj: the neighbour's code is
        // that column's), so exactly one change point p in (b, hi]: the
        // first column whose code exceeds `code`.  p = be: no change inside.
        int lo = b + 1, hi = min(be, nj - 1);
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (perp_code<MINPOS>(A, R, colx[mid], c, rech) > code) hi = mid; else lo = mid + 1;
        }
        if (lo >= be) {
          if (code >= 0 && code < n1) add_sums<COORD>(A, d, R, k, code, be - b, ewd - pwd.x, ew - pwd.y, el - pl, acc);
        } else {
          const double4 pp = pre[lo];
          if (code >= 0 && code < n1) add_sums<COORD>(A, d, R, k, code, lo - b, pp.x - pwd.x, pp.y - pwd.y, pp.z - pl, acc);
          if (ce >= 0 && ce < n1) add_sums<COORD>(A, d, R, k, ce, be - lo, ewd - pp.x, ew - pp.y, el - pp.z, acc);
        }
      } else {
        do_run_from<COORD, MINPOS>(A, d, colx, pre, c, R, k, b, be, code, acc, rech);
      }
    }
    b = nb;
    nb = nnb;
    x2 = nx2;
    pwd = npwd;
    pl = npl;
    cR = nR;
  }
  if (owner) acc.finish<COORD>(A, d, k);
  stats[0] += n_eval;
  stats[1] += rech;
}

// The arguments stay in the kernel's parameter space (__grid_constant__):
// the inlined sweep reads them as constant-bank operands, and the rarely
// called out-of-line helpers take them by reference without a copy.
template <int COORD, bool MINPOS>
__global__ void __launch_bounds__(kGridThreads, 4) grid_kernel(const __grid_constant__ PairArgs A) {
  __shared__ double prev[8 * kGridThreads];  // GridAcc's sums of code C - 1, per lane
  const int lane = threadIdx.x & 31;
  unsigned long long stats[2] = {0ull, 0ull};  // evaluated pairs, FP64 re-evaluations
  unsigned long long n_taken = 0;
  const int n0 = (int)A.g.n0;
  const float tmax = A.thr[n0];  // fl|x1 - x2| >= tmax: rejected by the first axis
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(A.next_item, 1ull);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= A.n_items) break;
    SweepItem it;
    if (!load_item<COORD>(A, idx, tmax, it)) continue;  // another kernel's item
    if (!grid_item(A, it.i, it.j)) continue;             // the pointer sweep's item
    ++n_taken;
    if (it.r_hi <= it.r_lo) continue;
    const int fi = (int)A.gfirst[it.i], fj = (int)A.gfirst[it.j];
    for (int t0 = 0; t0 < 2 * n0 + 1; t0 += kPassRuns)
      grid_pass<COORD, MINPOS>(A, it, fi, fj, t0, min(kPassRuns, 2 * n0 + 1 - t0), lane, prev + threadIdx.x,
                               stats);
  }
  add_counters(A, lane, stats[0], stats[1], n_taken, 9);
}

// Persistent launch: `ctas_per_sm` CTAs per SM (0 or above the occupancy
// limit: as many as fit), or with `max_out` set only that limit.
template <int COORD, bool MINPOS>
cudaError_t launch_grid(const PairArgs& a, int num_sms, int ctas_per_sm, cudaStream_t stream, int* max_out) {
  int per_sm = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, grid_kernel<COORD, MINPOS>, kGridThreads, 0);
  if (e != cudaSuccess) return e;
  per_sm = std::max(per_sm, 1);
  if (max_out) {
    *max_out = per_sm;
    return cudaSuccess;
  }
  if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
  grid_kernel<COORD, MINPOS><<<num_sms * per_sm, kGridThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_grid_kernel(const PairArgs& a, int coord, bool minpos, int num_sms, int ctas_per_sm,
                               cudaStream_t stream, int* max_out) {
  if (coord == TOS_CARTESIAN)
    return minpos ? launch_grid<kCart, true>(a, num_sms, ctas_per_sm, stream, max_out)
                  : launch_grid<kCart, false>(a, num_sms, ctas_per_sm, stream, max_out);
  return minpos ? launch_grid<kObs, true>(a, num_sms, ctas_per_sm, stream, max_out)
                : launch_grid<kObs, false>(a, num_sms, ctas_per_sm, stream, max_out);
}

}  // namespace tos
