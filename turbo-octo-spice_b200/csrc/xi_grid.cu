// xi_grid.cu — grid-sweep kernel of the XiEstimator pair count (Cartesian
// and observing coordinates) for catalogues whose first-axis coordinate takes
// few distinct values: forests on a common log-wavelength grid, whose
// distances are one function of loglam (h5healxi.cc:196-203).
//
// With U the sorted distinct first-axis values of the catalogue and a
// sightline contiguous on U (its pixel p has value U[f + p]), the run
// boundaries of xi_sweep.cuh for a row x1 = U[g] along any column sightline j
// are
//   q_k = clamp(Q[side][g][k] - f_j, 0, n_j),
// where Q[side][g][k] is the first grid index g2 whose value passes the
// boundary predicate of threshold T[k] against U[g].  Q is built once per
// call (k_grid_table, engine.cu), so a lane reads both ends of its run with
// two adjacent table loads instead of walking pointers.
#include "xi_sweep.cuh"

namespace tos {
namespace {

constexpr int kGridWarps = 4;  // warps per CTA of the grid-sweep kernel

// Rows [r_lo, r_hi) of an item for the (side, bin) tasks t0 .. t0 + m - 1
// (m = min(32, tasks left)).  A group of m < 32 tasks splits the rows into
// P = 32 / m phases: lane = task + m * phase takes rows r_lo + phase + P i,
// so the last, partial group of a grid costs 1/P of a full pass.
template <int COORD, bool MINPOS>
__device__ __noinline__ void grid_group(const PairArgs& A, const SweepItem& it, int fi, int fj,
                                        int t0, int lane, unsigned long long* stats) {
  const int n0 = (int)A.g.n0;
  const int m = min(32, 2 * n0 - t0);
  const int P = 32 / m;
  const bool act = lane < m * P;
  const int task = t0 + (act ? lane % m : 0);
  const int phase = act ? lane / m : 0;
  const int side = task / n0;
  const int k = task % n0;
  // the item in registers: the loop's flushes would force reloads from memory
  const int nj = it.nj, r_lo = it.r_lo, r_hi = it.r_hi;
  const Dest d = it.d;
  const double c = it.c;
  const float ap = it.ap, inv1sqf = A.inv1sqf;
  const float *rowd = it.rowd, *rowl = it.rowl, *roww = it.roww, *colx = it.colx;
  const double* rowwd = it.rowwd;
  const double4* pre = it.pre;
  const size_t qstride = (size_t)(n0 + 1);
  const uint16_t* qrow = A.gq + ((size_t)side * A.ng + fi) * qstride + k;
  RunAcc acc;
  acc.B = -1;
#pragma unroll
  for (int f = 0; f < 8; ++f) acc.s0[f] = acc.s1[f] = 0.0;
  unsigned rech = 0;
  unsigned long long n_eval = 0;
  // Rows where some task of the group has a non-empty run.  Table entries are
  // non-decreasing along the rows, so the run of (side, k) is non-empty on
  // one row interval: side 0 [Q_k, Q_k+1) needs Q_k+1 > fj and Q_k < fj + nj,
  // side 1 [Q_k+1, Q_k) needs Q_k > fj and Q_k+1 < fj + nj.
  int g_lo = r_hi, g_hi = r_lo;
  if (act) {
    const int lo_col = side ? 0 : 1, hi_col = side ? 1 : 0;
    int a = r_lo, b = r_hi;  // first row with Q[lo_col] > fj
    while (a < b) {
      const int mid = (a + b) >> 1;
      if ((int)qrow[(size_t)mid * qstride + lo_col] > fj) b = mid; else a = mid + 1;
    }
    int c2 = a, d2 = r_hi;  // first row with Q[hi_col] >= fj + nj
    while (c2 < d2) {
      const int mid = (c2 + d2) >> 1;
      if ((int)qrow[(size_t)mid * qstride + hi_col] >= fj + nj) d2 = mid; else c2 = mid + 1;
    }
    g_lo = a;
    g_hi = c2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    g_lo = min(g_lo, __shfl_xor_sync(kFull, g_lo, o));
    g_hi = max(g_hi, __shfl_xor_sync(kFull, g_hi, o));
  }
  if (g_hi <= g_lo) return;  // warp-uniform: every run of the group is empty
  // boundaries loaded one row ahead
  const int r0 = min(g_lo + phase, g_hi - 1);
  ushort2 nQ = make_ushort2(qrow[(size_t)r0 * qstride], qrow[(size_t)r0 * qstride + 1]);
  RowV nR = row_values<COORD>(rowd, rowwd, roww, rowl, ap, inv1sqf, r0);
#pragma unroll 1
  for (int r = g_lo + phase; r < g_hi; r += P) {
    const ushort2 Qv = nQ;
    const RowV R = nR;
    const int rn = min(r + P, g_hi - 1);
    nQ = make_ushort2(qrow[(size_t)rn * qstride], qrow[(size_t)rn * qstride + 1]);
    nR = row_values<COORD>(rowd, rowwd, roww, rowl, ap, inv1sqf, rn);
    const int qa = min(max((int)Qv.x - fj, 0), nj), qb = min(max((int)Qv.y - fj, 0), nj);
    const int s = side ? qb : qa, e = side ? qa : qb;
    if (act && e > s) {
      n_eval += (unsigned long long)(e - s);
      do_run<COORD, MINPOS>(A, d, colx, pre, c, R, k, s, e, acc, rech);
    }
  }
  if (act) {
    acc_flush8<COORD>(A, d, k, acc.B, acc.s0);
    acc_flush8<COORD>(A, d, k, acc.B + 1, acc.s1);
  }
  stats[0] += n_eval;
  stats[1] += rech;
}

template <int COORD, bool MINPOS>
__global__ void __launch_bounds__(kGridWarps * 32, 4) grid_kernel(PairArgs args) {
  // the arguments in shared memory: helpers take them by reference without a
  // per-thread local copy of the parameter block
  __shared__ PairArgs A;
  if (threadIdx.x == 0) A = args;
  __syncthreads();
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
    for (int t0 = 0; t0 < 2 * n0; t0 += 32) grid_group<COORD, MINPOS>(A, it, fi, fj, t0, lane, stats);
  }
  add_counters(A, lane, stats[0], stats[1], n_taken, 9);
}

// Persistent launch: as many CTAs as fit on the SMs at once.
template <int COORD, bool MINPOS>
cudaError_t launch_grid(const PairArgs& a, int num_sms, cudaStream_t stream) {
  int per_sm = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, grid_kernel<COORD, MINPOS>, kGridWarps * 32, 0);
  if (e != cudaSuccess) return e;
  grid_kernel<COORD, MINPOS><<<num_sms * (per_sm > 0 ? per_sm : 1), kGridWarps * 32, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_grid_kernel(const PairArgs& a, int coord, bool minpos, int num_sms,
                               cudaStream_t stream) {
  if (coord == TOS_CARTESIAN)
    return minpos ? launch_grid<kCart, true>(a, num_sms, stream)
                  : launch_grid<kCart, false>(a, num_sms, stream);
  return minpos ? launch_grid<kObs, true>(a, num_sms, stream) : launch_grid<kObs, false>(a, num_sms, stream);
}

}  // namespace tos
