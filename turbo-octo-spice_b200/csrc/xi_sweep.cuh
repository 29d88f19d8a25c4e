// xi_sweep.cuh — the run sweep shared by the grid-sweep kernel (xi_grid.cu,
// bin boundaries read from a table of the catalogue's common coordinate grid)
// and the pointer-sweep kernel (xi_runs.cu, boundaries found by walking
// column pointers): Cartesian (r_par, r_perp) and observing (dloglam, theta)
// coordinates, items whose z index is constant.
//
// For one sightline pair (i, j) with both sightlines sorted, fix a row p1 of
// i.  Along the columns p2 of j the reference's first-axis value is the float
// |x1 - x2| (XiEstimator.cc:242, 280) and its bin ref_u32((r - min) * inv)
// (XiEstimator.cc:243, 280) is a non-decreasing step function of that float.
// With the exact float thresholds
//   T[k] = smallest float r whose first-axis code is >= k   (k = 0..n0)
// the columns of bin k form one run on each side of x1:
//   side 0 (x2 >= x1): [q_k, q_k+1),  q_k = first p2 with x2 >= x1 and fl(x2 - x1) >= T[k]
//   side 1 (x2 <  x1): [q_k+1, q_k),  q_k = first p2 with x2 >= x1 or  fl(x1 - x2) <  T[k]
// so a lane that owns one (side, bin) task decides the first-axis bin of
// every pixel pair of a row from two boundaries, without visiting the pairs.
//
// Cartesian r_perp (XiEstimator.cc:246-248) is non-decreasing in x2 along a
// row (the host verifies that the FP64 rounding of the reference's expression
// cannot reorder pixels across a bin edge), so the r_perp code is evaluated
// at the two ends of a run only, in FP32 with an FP64 re-evaluation within
// 2^-K bins of an edge (the pixel-pair kernel's decision, xi_kernels.cu
// fast_bin), and a run whose ends differ is split by bisection.
//
// A sub-run [s, e) of row p1 contributes m = e - s pairs and, through the
// FP64 prefix sums P of sightline j, the XiBin sums
//   didj += wd1 * (P_wd[e] - P_wd[s]),  di += wd1 * m,  dj += P_wd[e] - P_wd[s],
//   wgt  += w1  * (P_w[e]  - P_w[s]),   wi += w1 * m,   wj += P_w[e]  - P_w[s],
//   z    += 0.5 * (l1 * m + P_l[e] - P_l[s])            (types.h:77-87),
// summed in FP64 registers of the lane (two consecutive r_perp codes at a
// time) over the rows and added to the per-cell 128-bit fixed-point sums
// when the lane's codes move on.
#pragma once

#include "xi_device.cuh"

namespace tos {
namespace {

// Where an item's sums go.
struct Dest {
  uint32_t cell, zb, sep;
};

// Seven XiBin sums and a pair count (passed by value to the flush).
struct FAcc {
  double s[7];
  unsigned int n;
  int code;
};

// Add (s, n) to bin (k, c) of the item's cell.
template <int COORD>
__device__ __forceinline__ void add_bin(const PairArgs& A, Dest d, int k, int c, const FAcc& F) {
  const uint32_t b = (COORD == kObs) ? d.sep + (uint32_t)k * A.g.n1 : (uint32_t)c + (uint32_t)k * A.g.n1;
  const uint32_t idx = d.zb + b * A.g.n2;  // unchecked, as XiEstimator.cc:249-254, 283-288
  if (idx >= A.g.ntotal) {
    atomicAdd(&A.counters[2], (unsigned long long)F.n);
    return;
  }
  unsigned long long* base = A.acc + ((size_t)d.cell * A.g.ntotal + idx) * kAccWords;
#pragma unroll
  for (int f = 0; f < 7; ++f) add128(base + f, base + 7 + f, to_fixed_wide(F.s[f], A.scale_hi[f]));
  red_add(base + 14, (unsigned long long)F.n);
}

// Exact r_perp code of a pair: -1 below the axis, 0..n1-1, n1 above
// (XiEstimator.cc:246-248 in the reference's FP64 expression order).
__device__ __noinline__ int exact_perp_code(float d1, float d2, double c, const RefGrid& g) {
  const double r1_sq = (double)fmul(d1, d1);
  const double two_r1_cos12 = dmul((double)fmul(2.0f, d1), c);
  const double r_para = (double)fabsf(fsub(d1, d2));
  const double r_sq = dadd(r1_sq, dmul(dsub((double)d2, two_r1_cos12), (double)d2));
  const double x = fabs(dsub(r_sq, dmul(r_para, r_para)));
  const double t = dmul(dsub(dsqrt(x), g.min1), g.inv1);
  if (!(t > -1.0)) return -1;
  const uint32_t q = ref_u32(t);
  return q >= g.n1 ? (int)g.n1 : (int)q;
}

// Row values: distance, the Cartesian u = |A1 * d2 + dl1| ~ (r_perp inv1)^2
// constants, and the pair-sum factors.
struct RowV {
  float d1, A1, dl1;
  double wd1, w1, hl1;
};

// r_perp code of column value x2 for row R (FP32, FP64 near an edge).
template <bool MINPOS>
__device__ __forceinline__ int perp_code(const PairArgs& A, const RowV& R, float x2, double c,
                                         unsigned& rech) {
  const float u = fabsf(__fmaf_rn(R.A1, x2, R.dl1));
  const float t1 = __fadd_rn(sqrt_approx(u), A.off1f);
  const int q1 = __float_as_int(__fadd_rz(t1, A.mag1)) - A.bits1;
  const bool edge =
      (((q1 + 1) & ((1 << A.k1) - 1)) < 2) && (t1 < A.n1p1f) && (!MINPOS || t1 > -2.0f);
  int code;
  if (!(t1 < A.n1f))
    code = (int)A.g.n1;
  else if (MINPOS && !(t1 > -1.0f))
    code = -1;
  else
    code = max(q1 >> A.k1, 0);
  if (edge) {
    ++rech;
    code = exact_perp_code(R.d1, x2, c, A.g);
  }
  return code;
}

// Per-lane FP64 sums of two consecutive r_perp codes B and B + 1 of one
// first-axis bin (7 XiBin sums and the pair count).
struct RunAcc {
  int B;
  double s0[8], s1[8];
  template <int COORD>
  __device__ __forceinline__ void add(const PairArgs& A, Dest d, int k, int cc, const double (&v)[8]);
};

// Add one code's sums of first-axis bin k to the per-cell sums (by value, so
// that the lane's accumulators stay in registers).
template <int COORD>
__device__ __noinline__ void acc_flush(const PairArgs& A, Dest d, int k, int c, FAcc F) {
  if (F.n == 0u) return;
  add_bin<COORD>(A, d, k, c, F);
}

template <int COORD>
__device__ __forceinline__ void acc_flush8(const PairArgs& A, Dest d, int k, int c,
                                           const double (&v)[8]) {
  FAcc F;
#pragma unroll
  for (int f = 0; f < 7; ++f) F.s[f] = v[f];
  F.n = (unsigned int)v[7];
  F.code = c;
  acc_flush<COORD>(A, d, k, c, F);
}

// Add sums v of r_perp code cc to the lane's two FP64 code accumulators.
template <int COORD>
__device__ __forceinline__ void add_vals(const PairArgs& A, Dest d, int k, int cc, const double (&v)[8],
                                         RunAcc& acc) {
  if (acc.B < 0) acc.B = cc;
  if (cc == acc.B) {
#pragma unroll
    for (int f = 0; f < 8; ++f) acc.s0[f] += v[f];
  } else if (cc == acc.B + 1) {
#pragma unroll
    for (int f = 0; f < 8; ++f) acc.s1[f] += v[f];
  } else if (cc == acc.B + 2) {
    acc_flush8<COORD>(A, d, k, acc.B, acc.s0);
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      acc.s0[f] = acc.s1[f];
      acc.s1[f] = v[f];
    }
    acc.B += 1;
  } else if (cc > acc.B + 2) {
    acc_flush8<COORD>(A, d, k, acc.B, acc.s0);
    acc_flush8<COORD>(A, d, k, acc.B + 1, acc.s1);
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      acc.s0[f] = v[f];
      acc.s1[f] = 0.0;
    }
    acc.B = cc;
  } else {
    acc_flush8<COORD>(A, d, k, cc, v);  // below the accumulator's codes: straight out
  }
}

template <int COORD>
__device__ __forceinline__ void RunAcc::add(const PairArgs& A, Dest d, int k, int cc, const double (&v)[8]) {
  add_vals<COORD>(A, d, k, cc, v, *this);
}

// Add a sub-run of m columns with r_perp code cc of first-axis bin k, given
// the differences of sightline j's prefix sums over it (w*delta, w, loglam),
// to the lane's code accumulators (RunAcc, or the grid sweep's GridAcc).
template <int COORD, class Acc>
__device__ __forceinline__ void add_sums(const PairArgs& A, Dest d, const RowV& R, int k, int cc, int m,
                                         double dwd, double dw, double dl, Acc& acc) {
  double v[8];
  const double md = (double)m;
  v[0] = R.wd1 * dwd;
  v[1] = R.wd1 * md;
  v[2] = dwd;
  v[3] = R.w1 * dw;
  v[4] = R.w1 * md;
  v[5] = dw;
  v[6] = __fma_rn(R.hl1, md, 0.5 * dl);
  v[7] = md;
  acc.template add<COORD>(A, d, k, cc, v);
}

// Add the sub-run [s, e) with r_perp code cc of first-axis bin k.
template <int COORD, class Acc>
__device__ __forceinline__ void add_subrun(const PairArgs& A, Dest d, const double4* pre,
                                           const RowV& R, int k, int cc, int s, int e,
                                           Acc& acc) {
  const double4 ps = pre[s], pe = pre[e];
  add_sums<COORD>(A, d, R, k, cc, e - s, pe.x - ps.x, pe.y - ps.y, pe.z - ps.z, acc);
}

// One run [s, e) of first-axis bin k in row R whose first column has r_perp
// code `code`: split by r_perp code (the code at the run's end; bisection
// between the ends when they differ) and add.
template <int COORD, bool MINPOS, class Acc>
__device__ __forceinline__ void do_run_from(const PairArgs& A, Dest d, const float* colx,
                                            const double4* pre, double c, const RowV& R, int k, int s,
                                            int e, int code, Acc& acc, unsigned& rech) {
  const int ce = (e - 1 == s) ? code : perp_code<MINPOS>(A, R, colx[e - 1], c, rech);
  const int n1 = (int)A.g.n1;
  if (code == ce) {  // one r_perp bin over the whole run
    if (code >= 0 && code < n1) add_subrun<COORD>(A, d, pre, R, k, code, s, e, acc);
    return;
  }
  int start = s;
  for (int guard = 0; guard <= n1 + 2; ++guard) {
    int end;
    if (code >= ce) {
      end = e;
    } else {
      // first p in (start, e - 1] whose code exceeds `code` (code(e-1) = ce does)
      int lo = start + 1, hi = e - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (perp_code<MINPOS>(A, R, colx[mid], c, rech) > code)
          hi = mid;
        else
          lo = mid + 1;
      }
      end = lo;
    }
    if (code >= 0 && code < n1) add_subrun<COORD>(A, d, pre, R, k, code, start, end, acc);
    if (end >= e) break;
    start = end;
    code = perp_code<MINPOS>(A, R, colx[end], c, rech);
  }
}

// One run [s, e) of first-axis bin k in row R: split by r_perp code (codes at
// the run's ends; bisection between them when they differ) and add.
template <int COORD, bool MINPOS>
__device__ __forceinline__ void do_run(const PairArgs& A, Dest d, const float* colx,
                                       const double4* pre, double c, const RowV& R, int k, int s,
                                       int e, RunAcc& acc, unsigned& rech) {
  if (COORD == kObs) {
    add_subrun<COORD>(A, d, pre, R, k, 0, s, e, acc);
    return;
  }
  const int code = perp_code<MINPOS>(A, R, colx[s], c, rech);
  do_run_from<COORD, MINPOS, RunAcc>(A, d, colx, pre, c, R, k, s, e, code, acc, rech);
}

// first p in [lo, n) with pred(col[p]); pred monotone
template <class Pred>
__device__ __forceinline__ int bsearch_col(const float* col, int lo, int n, Pred pred) {
  int hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pred(col[mid]))
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// Boundary predicate of threshold t (monotone in the column value x2):
//   side 0: x2 >= x1 and fl(x2 - x1) >= t;  side 1: x2 >= x1 or fl(x1 - x2) < t
__device__ __forceinline__ bool ptr_pred(int side, float x1, float x2, float t) {
  const bool ge = x2 >= x1;
  return side ? (ge || !(__fsub_rn(x1, x2) >= t)) : (ge && __fsub_rn(x2, x1) >= t);
}

// An item of a run-sweep kernel: rows of sightline i, columns of sightline j.
struct SweepItem {
  uint32_t i, j;
  int ni, nj, r_lo, r_hi;
  Dest d;
  double c;
  float ap;  // Cartesian: 2 (1 - c) inv1^2
  const float *rowd, *rowl, *rowx, *roww, *colx;
  const double* rowwd;
  const double4* pre;
  const PixPack* rowp;  // padded (distance, weight, w*delta) of the rows
};

// Load work item idx; false when the item belongs to another kernel (z index
// not constant over it, or run_item() rejects it) or has no rows that reach
// the columns ([r_lo, r_hi): fl(col_min - x1) < T[n0], fl(x1 - col_max) < T[n0]).
template <int COORD>
__device__ __forceinline__ bool load_item(const PairArgs& A, unsigned long long idx, float tmax,
                                          SweepItem& it) {
  it.i = A.item_i[idx];
  it.j = A.item_j[idx];
  it.ni = (int)A.npix[it.i];
  it.nj = (int)A.npix[it.j];
  if (it.ni == 0 || it.nj == 0) return false;
  const float4 ri = A.range[it.i], rj = A.range[it.j];
  const float lsum_lo = __fadd_rn(ri.z, rj.z), lsum_hi = __fadd_rn(ri.w, rj.w);
  const double zlo = dmul(dsub(dmul(0.5, (double)lsum_lo), A.g.min2), A.g.invn2);
  const double zhi = dmul(dsub(dmul(0.5, (double)lsum_hi), A.g.min2), A.g.invn2);
  it.d.zb = zbin_of_sum(lsum_lo, A.g);
  const bool zconst = zlo > -1.0 && zhi < 2147483648.0 && it.d.zb == zbin_of_sum(lsum_hi, A.g);
  it.c = A.item_c[idx];
  if (!run_item(A, it.c, zconst)) return false;
  it.d.cell = dest_row(A, it.i, it.j);
  it.d.sep = (COORD == kObs) ? A.item_sep[idx] : 0u;
  const uint64_t oi = A.off[it.i] + (uint64_t)kPad * (it.i + 1);
  const uint64_t oj = A.off[it.j] + (uint64_t)kPad * (it.j + 1);
  it.rowd = A.dist_pad + oi;
  it.rowp = A.pack + oi;
  it.rowl = A.loglam_pad + oi;
  it.rowx = (COORD == kObs) ? it.rowl : it.rowd;
  it.rowwd = A.wd + A.off[it.i];
  it.roww = A.w + A.off[it.i];
  it.colx = (COORD == kObs) ? A.loglam_pad + oj : A.dist_pad + oj;
  it.pre = A.prefix + A.off[it.j] + it.j;
  const float cmin = (COORD == kObs) ? rj.z : rj.x, cmax = (COORD == kObs) ? rj.w : rj.y;
  const double a = 2.0 * dsub(1.0, it.c);
  it.ap = (float)(a * A.g.inv1 * A.g.inv1);
  it.r_lo = bsearch_col(it.rowx, 0, it.ni, [&](float x1) { return __fsub_rn(cmin, x1) < tmax; });
  it.r_hi = bsearch_col(it.rowx, it.r_lo, it.ni, [&](float x1) { return __fsub_rn(x1, cmax) >= tmax; });
  return true;
}

// The loaded values of row r of an item (loaded a row ahead by the grid
// sweep) and the row values derived from them.
struct RowRaw {
  float d1, w1, l1;
  double wd1;
};

__device__ __forceinline__ RowRaw row_raw(const float* rowd, const double* rowwd, const float* roww,
                                          const float* rowl, int r) {
  RowRaw q;
  q.d1 = rowd[r];
  q.wd1 = rowwd[r];
  q.w1 = roww[r];
  q.l1 = rowl[r];
  return q;
}

// The same from the packed row array (one 16-byte load and the loglam).
__device__ __forceinline__ RowRaw row_raw_packed(const PixPack* rowp, const float* rowl, int r) {
  const PixPack p = rowp[r];
  RowRaw q;
  q.d1 = p.d;
  q.wd1 = p.wd;
  q.w1 = p.w;
  q.l1 = rowl[r];
  return q;
}

template <int COORD>
__device__ __forceinline__ RowV row_derive(const RowRaw& q, float ap, float inv1sqf) {
  RowV R;
  R.d1 = q.d1;
  R.wd1 = q.wd1;
  R.w1 = (double)q.w1;
  R.hl1 = 0.5 * (double)q.l1;
  if (COORD == kCart) {
    const float p = __fmul_rn(R.d1, R.d1);
    const float err = __fmaf_rn(R.d1, R.d1, -p);  // d1*d1 = p + err exactly
    R.A1 = __fmul_rn(R.d1, ap);
    R.dl1 = __fmul_rn(-err, inv1sqf);
  } else {
    R.A1 = R.dl1 = 0.f;
  }
  return R;
}

// Row r of an item.
template <int COORD>
__device__ __forceinline__ RowV row_values(const float* rowd, const double* rowwd, const float* roww,
                                           const float* rowl, float ap, float inv1sqf, int r) {
  return row_derive<COORD>(row_raw(rowd, rowwd, roww, rowl, r), ap, inv1sqf);
}

// Warp-sum the kernel's counters into A.counters[0] (evaluated pairs), [1]
// (FP64 re-evaluations) and [slot] (items taken).
__device__ __forceinline__ void add_counters(const PairArgs& A, int lane, unsigned long long n_eval,
                                             unsigned long long n_recheck, unsigned long long n_taken,
                                             int slot) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_eval += __shfl_xor_sync(kFull, n_eval, o);
    n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  }
  if (lane == 0) {
    atomicAdd(&A.counters[0], n_eval);
    atomicAdd(&A.counters[1], n_recheck);
    atomicAdd(&A.counters[slot], n_taken);
  }
}

}  // namespace
}  // namespace tos
