// xi_diag.cu — diagonal-sweep kernel of the XiEstimator pair count for Polar
// (r, mu) coordinates (XiEstimator.cc:168-225), items whose z index is
// constant.
//
// Along a row of the pixel-pair matrix the Polar key (r bin, mu bin) changes
// every few columns, so runs along rows are short.  Along a diagonal
// (p1 + s, p2 + s) both distances grow together: r_par = d2 - d1 stays nearly
// constant and r_perp grows slowly, so the key stays the same for tens to
// hundreds of pairs.  A lane therefore owns one diagonal p2 - p1 = delta of
// an item and walks it row by row: every pair is binned (FP32, with an FP64
// re-evaluation of the reference's expression near an edge, as in the
// pixel-pair kernel), and while the key stays the same the lane only adds
// the two pair products w_i d_i w_j d_j and w_i w_j in FP64 registers.  The
// other XiBin sums of a run of rows [s0, s1) on diagonal delta are
// differences of the two sightlines' FP64 prefix sums:
//   di = P_i[s1] - P_i[s0],  dj = P_j[s1 + delta] - P_j[s0 + delta]  (w d, w, loglam).
// When the key changes the run's sums go, as fixed-point values, to the
// per-cell 128-bit sums.  The 32 lanes of a warp own 32 consecutive
// diagonals, so a step reads one row value (broadcast) and 32 consecutive
// column values.
#include "xi_device.cuh"

namespace tos {
namespace {

constexpr int kDiagWarps = 8;  // warps per CTA

// Row values of the pixel-pair kernel's Polar fast path (xi_kernels.cu
// fast_bin): x1 = d1, A1 = d1 * 2(1 - c), dl1 = -(d1*d1 - fl(d1*d1)).
struct DRow {
  float x1, d1, A1, dl1;
};

// FP32 Polar key of one pixel pair (packed b0 << 16 | b1, or kInvalidKey) and
// whether it lies within 2^-K bins of an edge (or r^2 is tiny) and must be
// re-binned in FP64.  The same decision as xi_kernels.cu fast_bin.
template <bool MINPOS>
__device__ __forceinline__ uint32_t polar_key(const PairArgs& A, const DRow& R, float x2, bool& recheck) {
  const float s = __fsub_rn(x2, R.x1);
  const float r2 = __fmaf_rn(s, s, __fmaf_rn(R.A1, x2, R.dl1));
  const float rs = rsqrt_approx(r2);
  const float t0 = __fmaf_rn(__fmul_rn(r2, rs), A.inv0f, A.off0f);
  const float t1 = __fmaf_rn(__fmul_rn(fabsf(s), rs), A.inv1f, A.off1f);
  const bool small = !(r2 >= A.r2_small);
  const int q0 = __float_as_int(__fadd_rz(t0, A.mag0)) - A.bits0;
  const int q1 = __float_as_int(__fadd_rz(t1, A.mag1)) - A.bits1;
  bool valid = (t0 < A.n0f) && (t1 < A.n1f);
  bool coarse = (t0 < A.n0p1f) && (t1 < A.n1p1f);
  if (MINPOS) {
    valid = valid && (t0 > -1.0f) && (t1 > -1.0f);
    coarse = coarse && (t0 > -2.0f) && (t1 > -2.0f);
  }
  int b0 = q0 >> A.k0, b1 = q1 >> A.k1;
  if (MINPOS) {
    b0 = max(b0, 0);
    b1 = max(b1, 0);
  }
  const bool edge = (((q1 + 1) & ((1 << A.k1) - 1)) < 2) || (((q0 + 1) & ((1 << A.k0) - 1)) < 2);
  recheck = (coarse && edge) || small;
  return valid ? (((uint32_t)b0 << 16) | (uint32_t)b1) : kInvalidKey;
}

// Warp-sum the kernel's counters into A.counters[0] (evaluated pairs), [1]
// (FP64 re-evaluations) and [12] (items taken, the same count in every lane).
__device__ __forceinline__ void add_counters_diag(const PairArgs& A, int lane, unsigned long long n_eval,
                                                  unsigned long long n_recheck, unsigned long long n_taken) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_eval += __shfl_xor_sync(kFull, n_eval, o);
    n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  }
  if (lane == 0) {
    atomicAdd(&A.counters[0], n_eval);
    atomicAdd(&A.counters[1], n_recheck);
    atomicAdd(&A.counters[12], n_taken);
  }
}

// Per-item constants.
struct DItem {
  uint32_t cell, zb;
  int ni, nj;
  double c;
  float ap;  // 2(1 - c)
  const float* rowd;     // padded distances of sightline i
  const double* rowwd;   // w*delta of i
  const float* roww;     // w of i
  const double4* prei;   // prefix sums of i
  const float* cold;     // padded distances of sightline j
  const double* colwd;
  const float* colw;
  const double4* prej;
  const PixPack* rowp;   // padded (distance, weight, w*delta) of sightline i
  const PixPack* colp;   // the same of sightline j
};

// Add the run [s0, s1) of diagonal delta with key `key` to row `cell`
// (z index zb; prefix sums prei, prej of the item's two sightlines).
__device__ __noinline__ void emit_diag(const PairArgs& A, uint32_t cell, uint32_t zb, const double4* prei,
                                       const double4* prej, uint32_t key, int s0, int s1, int delta,
                                       double didj, double wgt) {
  const uint32_t b0 = key >> 16, b1 = key & 0xFFFFu;
  const uint32_t idx = zb + (b1 + b0 * A.g.n1) * A.g.n2;  // as XiEstimator.cc:196-201
  const unsigned long long m = (unsigned long long)(s1 - s0);
  if (idx >= A.g.ntotal) {
    atomicAdd(&A.counters[2], m);
    return;
  }
  const double4 ia = prei[s0], ib = prei[s1];
  const double4 ja = prej[s0 + delta], jb = prej[s1 + delta];
  double v[7];
  v[0] = didj;
  v[1] = ib.x - ia.x;
  v[2] = jb.x - ja.x;
  v[3] = wgt;
  v[4] = ib.y - ia.y;
  v[5] = jb.y - ja.y;
  v[6] = 0.5 * ((ib.z - ia.z) + (jb.z - ja.z));
  unsigned long long* base = A.acc + ((size_t)cell * A.g.ntotal + idx) * kAccWords;
#pragma unroll
  for (int f = 0; f < 7; ++f) add128(base + f, base + 7 + f, to_fixed_wide(v[f], A.scale_hi[f]));
  red_add(base + 14, m);
}

// A closed run of a diagonal, waiting in the warp's queue.
struct DRun {
  uint32_t key;
  int s0, s1, delta;
  double didj, wgt;
};
constexpr int kQueue = 64;  // runs per warp queue (drained 32 at a time)

// Emit the queue entries [first, first + n) of the warp, one per lane.
__device__ __forceinline__ void drain(const PairArgs& A, const DItem& it, const DRun* q, int first, int n,
                                      int lane) {
  __syncwarp();
  if (lane < n) {
    const DRun r = q[first + lane];
    emit_diag(A, it.cell, it.zb, it.prei, it.prej, r.key, r.s0, r.s1, r.delta, r.didj, r.wgt);
  }
  __syncwarp();
}

// Sweep diagonals delta0 .. delta0 + 31 (lane = delta - delta0) of an item
// over the rows [s_lo, s_hi) that reach one of them.  Lanes close runs at
// different rows, so a closed run goes to the warp's queue in shared memory
// and the warp emits 32 of them at a time, one per lane.
template <bool MINPOS>
__device__ __forceinline__ void diag_group(const PairArgs& A, const DItem& it, int delta0, int dhi, int lane,
                                           DRun* q, unsigned long long* stats) {
  const int delta = delta0 + lane;
  const bool lane_on = delta <= dhi;
  const int s_lo = max(0, -(delta0 + 31));
  const int s_hi = min(it.ni, it.nj - delta0);
  const unsigned lt = (1u << lane) - 1u;
  uint32_t cur = kInvalidKey;
  int s0 = 0;
  int qn = 0;  // queued runs (the same in every lane)
  double didj = 0.0, wgt = 0.0;
  unsigned rech = 0;
  unsigned n_eval = 0;  // at most one per row of the group
#pragma unroll 1
  for (int s = s_lo; s < s_hi; ++s) {
    // p2 stays within the 32 sentinels on either side of the padded
    // distances: p2 >= s_lo + delta0 >= -31 and p2 < s_hi + delta0 + 32 <= nj + 32
    const int p2 = s + delta;
    const bool in = lane_on && (unsigned)p2 < (unsigned)it.nj;
    // one 16-byte load each: the row's (broadcast) and the lane's column's
    // distance, weight and w*delta (padding: sentinel distance, zero weights)
    const PixPack rp = it.rowp[s], cq = it.colp[p2];
    DRow R;
    R.d1 = rp.d;
    R.x1 = R.d1;
    const float p = __fmul_rn(R.d1, R.d1);
    R.dl1 = -__fmaf_rn(R.d1, R.d1, -p);  // -(d1*d1 - fl(d1*d1)), exact
    R.A1 = __fmul_rn(R.d1, it.ap);
    const float x2 = cq.d;
    bool recheck;
    uint32_t key = polar_key<MINPOS>(A, R, x2, recheck);
    recheck = recheck && in;
    if (__any_sync(kFull, recheck)) {
      if (recheck) {
        uint32_t e0 = 0, e1 = 0;
        key = exact_polar(R.d1, x2, it.c, A.g, &e0, &e1) ? ((e0 << 16) | e1) : kInvalidKey;
        ++rech;
      }
    }
    if (!in) key = kInvalidKey;
    n_eval += in ? 1u : 0u;
    const bool change = key != cur;
    const bool close = change && cur != kInvalidKey;
    const unsigned cm = __ballot_sync(kFull, close);
    if (cm) {
      if (close) q[qn + __popc(cm & lt)] = DRun{cur, s0, s, delta, didj, wgt};
      qn += __popc(cm);
      if (qn >= 32) {
        qn -= 32;
        drain(A, it, q, qn, 32, lane);
      }
    }
    if (change) {
      cur = key;
      s0 = s;
      didj = 0.0;
      wgt = 0.0;
    }
    if (key != kInvalidKey) {  // binned: p2 is a pixel of sightline j
      didj = __fma_rn(rp.wd, cq.wd, didj);
      wgt = __fma_rn((double)rp.w, (double)cq.w, wgt);
    }
  }
  // runs still open at the last row, then the queue
  const bool close = cur != kInvalidKey;
  const unsigned cm = __ballot_sync(kFull, close);
  if (close) q[qn + __popc(cm & lt)] = DRun{cur, s0, s_hi, delta, didj, wgt};
  qn += __popc(cm);
  if (qn >= 32) {
    qn -= 32;
    drain(A, it, q, qn, 32, lane);
  }
  drain(A, it, q, 0, qn, lane);
  stats[0] += (unsigned long long)n_eval;
  stats[1] += rech;
}

// The arguments stay in the kernel's parameter space (__grid_constant__):
// the inlined sweep reads them as constant-bank operands, and emit_diag
// takes them by reference without a copy.
template <bool MINPOS>
__global__ void __launch_bounds__(kDiagWarps * 32, 3) diag_kernel(const __grid_constant__ PairArgs A) {
  __shared__ DRun queue[kDiagWarps][kQueue];
  const int lane = threadIdx.x & 31;
  DRun* q = queue[threadIdx.x >> 5];
  unsigned long long stats[2] = {0ull, 0ull};  // evaluated pairs, FP64 re-evaluations
  unsigned long long n_taken = 0;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(A.next_item, 1ull);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= A.n_items) break;
    const uint32_t i = A.item_i[idx], j = A.item_j[idx];
    const double c = A.item_c[idx];
    DItem it;
    it.ni = (int)A.npix[i];
    it.nj = (int)A.npix[j];
    if (it.ni == 0 || it.nj == 0) continue;
    const float4 ri = A.range[i], rj = A.range[j];
    const float lsum_lo = __fadd_rn(ri.z, rj.z), lsum_hi = __fadd_rn(ri.w, rj.w);
    const double zlo = dmul(dsub(dmul(0.5, (double)lsum_lo), A.g.min2), A.g.invn2);
    const double zhi = dmul(dsub(dmul(0.5, (double)lsum_hi), A.g.min2), A.g.invn2);
    it.zb = zbin_of_sum(lsum_lo, A.g);
    if (!diag_item(A, zlo, zhi, it.zb, zbin_of_sum(lsum_hi, A.g))) continue;  // the pixel-pair kernel's item
    ++n_taken;
    it.c = c;
    it.cell = dest_row(A, i, j);
    const double a = 2.0 * dsub(1.0, c);
    it.ap = (float)a;
    const uint64_t oi = A.off[i] + (uint64_t)kPad * (i + 1), oj = A.off[j] + (uint64_t)kPad * (j + 1);
    it.rowd = A.dist_pad + oi;
    it.cold = A.dist_pad + oj;
    it.rowwd = A.wd + A.off[i];
    it.roww = A.w + A.off[i];
    it.colwd = A.wd + A.off[j];
    it.colw = A.w + A.off[j];
    it.prei = A.prefix + A.off[i] + i;
    it.prej = A.prefix + A.off[j] + j;
    it.rowp = A.pack + oi;
    it.colp = A.pack + oj;
    // Column window |d1 - d2| < lim of every row (the pixel-pair kernel's
    // Polar bound: r^2 >= (d2 - d1)^2 + 2(1 - c) dmin_i dmin_j - err), and
    // from it the diagonals that reach it: delta in [dlo, dhi].
    float lim = A.win_lim;
    if (A.prune && ri.x > 0.f && rj.x > 0.f) {
      const double q = A.polar_r2 - fmax(a, 0.0) * (double)ri.x * (double)rj.x * (1.0 - 1e-6) + A.polar_e2;
      lim = fminf(lim, (float)(sqrt(fmax(q, 0.0)) * (1.0 + 1e-6) + 1e-3));
    }
    int dlo = 0x7FFFFFFF, dhi = -0x7FFFFFFF;
    if (!A.prune) {  // no window: every diagonal
      dlo = -(it.ni - 1);
      dhi = it.nj - 1;
    }
    for (int r = lane; A.prune && r < it.ni; r += 32) {
      const float x1 = it.rowd[r];
      int lo = 0, hi = it.nj;  // first column with fl(x1 - x2) < lim
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__fsub_rn(x1, it.cold[mid]) < lim) hi = mid; else lo = mid + 1;
      }
      int lo2 = lo, hi2 = it.nj;  // first column with x2 >= x1 and fl(x2 - x1) >= lim
      while (lo2 < hi2) {
        const int mid = (lo2 + hi2) >> 1;
        const float x2 = it.cold[mid];
        if (x2 >= x1 && __fsub_rn(x2, x1) >= lim) hi2 = mid; else lo2 = mid + 1;
      }
      if (lo2 > lo) {
        dlo = min(dlo, lo - r);
        dhi = max(dhi, lo2 - 1 - r);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dlo = min(dlo, __shfl_xor_sync(kFull, dlo, o));
      dhi = max(dhi, __shfl_xor_sync(kFull, dhi, o));
    }
    for (int d0 = dlo; d0 <= dhi; d0 += 32) diag_group<MINPOS>(A, it, d0, dhi, lane, q, stats);
  }
  add_counters_diag(A, lane, stats[0], stats[1], n_taken);
}

// Persistent launch: `ctas_per_sm` CTAs per SM (0 or above the occupancy
// limit: as many as fit), or with `max_out` set only that limit.
template <bool MINPOS>
cudaError_t launch_diag(const PairArgs& a, int num_sms, int ctas_per_sm, cudaStream_t stream, int* max_out) {
  int per_sm = 0;
  const cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_kernel<MINPOS>, kDiagWarps * 32, 0);
  if (e != cudaSuccess) return e;
  per_sm = per_sm > 0 ? per_sm : 1;
  if (max_out) {
    *max_out = per_sm;
    return cudaSuccess;
  }
  if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
  diag_kernel<MINPOS><<<num_sms * per_sm, kDiagWarps * 32, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_diag_kernel(const PairArgs& a, bool minpos, int num_sms, int ctas_per_sm, cudaStream_t stream,
                               int* max_out) {
  return minpos ? launch_diag<true>(a, num_sms, ctas_per_sm, stream, max_out)
                : launch_diag<false>(a, num_sms, ctas_per_sm, stream, max_out);
}

}  // namespace tos
