// xi_runs.cu — pointer-sweep kernel of the XiEstimator pair count (Cartesian
// and observing coordinates): the run sweep of xi_sweep.cuh for sorted
// sightlines that are not contiguous on a common coordinate grid.
//
// A lane owns one (side, bin k) task and walks the rows with two column
// pointers, the first columns that pass the boundary predicates of T[k] and
// T[k+1].  Both predicates get harder as x1 grows, so the pointers only move
// right; the first row places them by binary search.  Each pointer keeps the
// column values around it in registers, so a step costs one load whose
// latency is hidden until the next step.
#include "xi_sweep.cuh"

namespace tos {
namespace {

constexpr int kRunWarps = 4;  // warps per CTA of the pointer-sweep kernel

// A column pointer with prev = colx[p - 1], cur = colx[p], next = colx[p + 1]
// (the padding of the column array keeps p - 1 and p + 1 in bounds for
// 0 <= p <= nj).
struct ColPtr {
  int p;
  float prev, cur, next;
  __device__ __forceinline__ void init(const float* colx, int q) {
    p = q;
    prev = colx[q - 1];
    cur = colx[q];
    next = colx[q + 1];
  }
  __device__ __forceinline__ void step(const float* colx) {
    ++p;
    prev = cur;
    cur = next;
    next = colx[p + 1];
  }
  // first column at or after p passing pred(x1, ., t)
  __device__ __forceinline__ void advance(const float* colx, int nj, int side, float x1, float t) {
    while (p < nj && !ptr_pred(side, x1, cur, t)) step(colx);
  }
};

// Rows [r_lo, r_hi) of an item for the (side, bin) tasks t0 .. t0 + m - 1
// (m = min(32, tasks left)); a partial group splits the rows into P = 32 / m
// phases, lane = task + m * phase taking rows r_lo + phase + P i (the
// pointers still only move right).
template <int COORD, bool MINPOS>
__device__ __noinline__ void run_group(const PairArgs& A, const SweepItem& it, int t0, int lane,
                                       unsigned long long* stats) {
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
  const float *rowd = it.rowd, *rowl = it.rowl, *roww = it.roww, *rowx = it.rowx, *colx = it.colx;
  const double* rowwd = it.rowwd;
  const double4* pre = it.pre;
  const float ta = A.thr[k], tb = A.thr[k + 1];
  const float x1f = rowx[min(r_lo + phase, r_hi - 1)];
  ColPtr pa, pb;
  pa.init(colx, bsearch_col(colx, 0, nj, [&](float x2) { return ptr_pred(side, x1f, x2, ta); }));
  pb.init(colx, bsearch_col(colx, 0, nj, [&](float x2) { return ptr_pred(side, x1f, x2, tb); }));
  RunAcc acc;
  acc.B = -1;
#pragma unroll
  for (int f = 0; f < 8; ++f) acc.s0[f] = acc.s1[f] = 0.0;
  unsigned rech = 0;
  unsigned long long n_eval = 0;
#pragma unroll 1
  for (int r = r_lo + phase; r < r_hi; r += P) {
    const float x1 = rowx[r];
    if (!act) continue;
    pa.advance(colx, nj, side, x1, ta);
    pb.advance(colx, nj, side, x1, tb);
    const int s = side ? pb.p : pa.p, e = side ? pa.p : pb.p;
    if (e > s) {
      n_eval += (unsigned long long)(e - s);
      const RowV R = row_values<COORD>(rowd, rowwd, roww, rowl, ap, inv1sqf, r);
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
__global__ void __launch_bounds__(kRunWarps * 32, 4) run_kernel(PairArgs args) {
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
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(A.next_item, (unsigned long long)kClaimItems);
    base = __shfl_sync(kFull, base, 0);
    if (base >= A.n_items) break;
    const unsigned long long mine = base + lane;
    unsigned todo = __ballot_sync(kFull, mine < A.n_items && item_owner(A, mine) == kOwnerRun);
    while (todo) {
      const unsigned long long idx = base + (__ffs(todo) - 1);
      todo &= todo - 1;
      SweepItem it;
      if (!load_item<COORD>(A, idx, tmax, it)) continue;  // another kernel's item
      if (grid_item(A, it.i, it.j)) continue;              // the grid sweep's item
      ++n_taken;
      if (it.r_hi <= it.r_lo) continue;
      for (int t0 = 0; t0 < 2 * n0; t0 += 32) run_group<COORD, MINPOS>(A, it, t0, lane, stats);
    }
  }
  add_counters(A, lane, stats[0], stats[1], n_taken, 8);
}

// Persistent launch: as many CTAs as fit on the SMs at once.
template <int COORD, bool MINPOS>
cudaError_t launch_run(const PairArgs& a, int num_sms, cudaStream_t stream) {
  int per_sm = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, run_kernel<COORD, MINPOS>, kRunWarps * 32, 0);
  if (e != cudaSuccess) return e;
  run_kernel<COORD, MINPOS><<<num_sms * (per_sm > 0 ? per_sm : 1), kRunWarps * 32, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_run_kernel(const PairArgs& a, int coord, bool minpos, int num_sms,
                              cudaStream_t stream) {
  if (coord == TOS_CARTESIAN)
    return minpos ? launch_run<kCart, true>(a, num_sms, stream)
                  : launch_run<kCart, false>(a, num_sms, stream);
  return minpos ? launch_run<kObs, true>(a, num_sms, stream) : launch_run<kObs, false>(a, num_sms, stream);
}

}  // namespace tos
