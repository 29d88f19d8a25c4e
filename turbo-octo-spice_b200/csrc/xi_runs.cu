// xi_runs.cu — run-sweep kernel of the XiEstimator pair count for Cartesian
// (r_par, r_perp) and observing (dloglam, theta) coordinates.
//
// For one sightline pair (i, j) with both sightlines sorted, fix a row p1 of
// i.  Along the columns p2 of j the reference's first-axis value is the float
// |x1 - x2| (XiEstimator.cc:242, 280), and its bin ref_u32((r - min) * inv)
// (XiEstimator.cc:243, 280) is a monotone step function of that float.  With
// the exact float thresholds
//   T[k] = smallest float r whose bin is >= k        (T[0]: first valid r)
// the columns holding bin k are one contiguous run on each side of x1:
//   right (x2 >= x1):  [Pr(T[k]), Pr(T[k+1])),  Pr(t) = first p2 with x2 >= x1 and fl(x2-x1) >= t
//   left  (x2 <  x1):  [Pl(T[k+1]), Pl(T[k])),  Pl(t) = first p2 with x2 >= x1 or  fl(x1-x2) <  t
// and every pointer only moves right as p1 grows.  A lane owns one (side, k)
// and walks the rows advancing its two pointers, so each pixel pair's first-
// axis bin is decided exactly without visiting the pair.
//
// Cartesian r_perp (XiEstimator.cc:246-248) grows monotonically with x2 along
// a run (the host verifies that its FP64 rounding noise cannot reorder pixels
// across any bin edge), so a run splits into at most a few r_perp sub-runs;
// the r_perp bin is evaluated only at sub-run ends, in FP32 with an FP64
// re-evaluation near an edge, and split points are found by bisection.
//
// A sub-run [s, e) of row p1 contributes m = e - s pairs and, through the
// FP64 prefix sums P of sightline j, the XiBin sums
//   didj += wd1 * (P_wd[e] - P_wd[s]),  di += wd1 * m,  dj += P_wd[e] - P_wd[s],
//   wgt  += w1  * (P_w[e]  - P_w[s]),   wi += w1 * m,   wj += P_w[e]  - P_w[s],
//   z    += 0.5 * (l1 * m + P_l[e] - P_l[s])            (types.h:77-87),
// accumulated in FP64 registers of the lane (two r_perp bins at a time) and
// added to the per-cell 128-bit fixed-point sums when the lane moves on.
#include "xi_device.cuh"

namespace tos {
namespace {

constexpr int kRunWarps = 4;  // warps per CTA of the run-sweep kernel

struct RRow {
  float x1;       // distance (or loglam)
  float d1;       // distance
  float A1, dl1;  // Cartesian: (r_perp * inv1)^2 = |A1 * d2 + dl1|
  double wd1, w1, hl1;
};

struct RItem {
  uint32_t i, j, ni, nj, cell, zb, sep;
  double c;
  float ap;  // Cartesian: 2 (1 - c) inv1^2
  const float* rowx;
  const float* rowd;
  const float* rowl;
  const double* rowwd;
  const float* roww;
  const float* colx;  // padded column coordinate of sightline j
  const double4* pre; // prefix sums of sightline j
  float col_min, col_max;
};

// Per-lane FP64 accumulator of two consecutive r_perp codes B and B+1.
struct RunAcc {
  int B;
  double s0[8], s1[8];  // 7 XiBin sums and the pair count
};

// Add one accumulator (code c of first-axis bin k) into the global sums.
template <int COORD>
__device__ void acc_flush(const PairArgs& A, const RItem& it, int k, int c, const double* s) {
  if (s[7] == 0.0) return;
  const uint32_t b =
      (COORD == kObs) ? it.sep + (uint32_t)k * A.g.n1 : (uint32_t)c + (uint32_t)k * A.g.n1;
  const uint32_t idx = it.zb + b * A.g.n2;
  const unsigned long long m = (unsigned long long)s[7];
  if (idx >= A.g.ntotal) {
    atomicAdd(&A.counters[2], m);
    return;
  }
  unsigned long long* base = A.acc + ((size_t)it.cell * A.g.ntotal + idx) * kAccWords;
#pragma unroll
  for (int f = 0; f < 7; ++f) add128(base + f, base + 7 + f, to_fixed_wide(s[f], A.scale_hi[f]));
  atomicAdd(base + 14, m);
}

// Exact r_perp code of a pair: -1 below the first valid value, 0..n1-1, n1 above
// (XiEstimator.cc:246-248 in the reference's FP64 expression order).
__device__ __forceinline__ int exact_perp_code(float d1, float d2, double c, const RefGrid& g) {
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

// r_perp code of column d2 (FP32 with FP64 re-evaluation near an edge).
template <bool MINPOS>
__device__ __forceinline__ int perp_code(const PairArgs& A, const RRow& R, double c, float d2,
                                         unsigned long long& n_recheck) {
  const float u = fabsf(__fmaf_rn(R.A1, d2, R.dl1));
  const float t1 = __fadd_rn(sqrt_approx(u), A.off1f);
  const int q1 = __float_as_int(__fadd_rz(t1, A.mag1)) - A.bits1;
  const bool edge =
      (((q1 + 1) & ((1 << A.k1) - 1)) < 2) && (t1 < A.n1p1f) && (!MINPOS || t1 > -2.0f);
  if (edge) {
    ++n_recheck;
    return exact_perp_code(R.d1, d2, c, A.g);
  }
  if (!(t1 < A.n1f)) return (int)A.g.n1;
  if (MINPOS && !(t1 > -1.0f)) return -1;
  return max(q1 >> A.k1, 0);
}

// Add the sub-run [s, e) with r_perp code cc of first-axis bin k.
template <int COORD>
__device__ __forceinline__ void add_subrun(const PairArgs& A, const RItem& it, const RRow& R,
                                           int k, int cc, int s, int e, RunAcc& acc) {
  const double4 ps = it.pre[s], pe = it.pre[e];
  const double md = (double)(e - s);
  const double dwd = pe.x - ps.x, dw = pe.y - ps.y, dl = pe.z - ps.z;
  double v[8];
  v[0] = R.wd1 * dwd;
  v[1] = R.wd1 * md;
  v[2] = dwd;
  v[3] = R.w1 * dw;
  v[4] = R.w1 * md;
  v[5] = dw;
  v[6] = __fma_rn(R.hl1, md, 0.5 * dl);
  v[7] = md;
  if (acc.B < 0) acc.B = cc;
  if (cc == acc.B) {
#pragma unroll
    for (int f = 0; f < 8; ++f) acc.s0[f] += v[f];
  } else if (cc == acc.B + 1) {
#pragma unroll
    for (int f = 0; f < 8; ++f) acc.s1[f] += v[f];
  } else if (cc == acc.B + 2) {
    acc_flush<COORD>(A, it, k, acc.B, acc.s0);
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      acc.s0[f] = acc.s1[f];
      acc.s1[f] = v[f];
    }
    acc.B += 1;
  } else if (cc > acc.B + 2) {
    acc_flush<COORD>(A, it, k, acc.B, acc.s0);
    acc_flush<COORD>(A, it, k, acc.B + 1, acc.s1);
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      acc.s0[f] = v[f];
      acc.s1[f] = 0.0;
    }
    acc.B = cc;
  } else {
    acc_flush<COORD>(A, it, k, cc, v);  // below the accumulator's codes: straight out
  }
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

// One run [s, e) of first-axis bin k in row R: split by r_perp code and add.
template <int COORD, bool MINPOS>
__device__ __forceinline__ void do_run(const PairArgs& A, const RItem& it, const RRow& R, int k,
                                       int s, int e, RunAcc& acc, unsigned long long& n_recheck) {
  if (COORD == kObs) {
    add_subrun<COORD>(A, it, R, k, 0, s, e, acc);
    return;
  }
  const int ce = perp_code<MINPOS>(A, R, it.c, it.colx[e - 1], n_recheck);
  int start = s;
  int code = (e - 1 == s) ? ce : perp_code<MINPOS>(A, R, it.c, it.colx[s], n_recheck);
  const int n1 = (int)A.g.n1;
  for (int guard = 0; guard <= n1 + 2; ++guard) {
    int end;
    if (code >= ce) {
      end = e;
    } else {
      // first p in (start, e - 1] whose code exceeds `code` (code(e-1) = ce does)
      int lo = start + 1, hi = e - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (perp_code<MINPOS>(A, R, it.c, it.colx[mid], n_recheck) > code)
          hi = mid;
        else
          lo = mid + 1;
      }
      end = lo;
    }
    if (code >= 0 && code < n1) add_subrun<COORD>(A, it, R, k, code, start, end, acc);
    if (end >= e) break;
    start = end;
    code = perp_code<MINPOS>(A, R, it.c, it.colx[end], n_recheck);
  }
}

template <int COORD, bool MINPOS>
__device__ void sweep_item(const PairArgs& A, const RItem& it, int lane, unsigned long long& n_eval,
                           unsigned long long& n_recheck) {
  const int n0 = (int)A.g.n0;
  const int nj = (int)it.nj;
  const int ntask = 2 * n0;
  const float tmax = A.thr[n0];  // fl|x1 - x2| >= tmax: rejected by the first axis
  // rows that can reach the columns: fl(col_min - x1) < tmax and fl(x1 - col_max) < tmax
  const float cmin = it.col_min, cmax = it.col_max;
  const int r_lo = bsearch_col(it.rowx, 0, (int)it.ni, [&](float x1) { return __fsub_rn(cmin, x1) < tmax; });
  const int r_hi =
      bsearch_col(it.rowx, r_lo, (int)it.ni, [&](float x1) { return __fsub_rn(x1, cmax) >= tmax; });
  if (r_hi <= r_lo) return;
  for (int g = 0; g * 32 < ntask; ++g) {
    const int task = g * 32 + lane;
    const bool act = task < ntask;
    const int side = act ? task / n0 : 0;  // 0: x2 >= x1, 1: x2 < x1
    const int k = act ? task % n0 : 0;
    const float ta = A.thr[k], tb = A.thr[k + 1];
    int pa = 0, pb = 0;
    RunAcc acc;
    acc.B = -1;
#pragma unroll
    for (int f = 0; f < 8; ++f) acc.s0[f] = acc.s1[f] = 0.0;
    for (int r = r_lo; r < r_hi; ++r) {
      RRow R;
      R.x1 = it.rowx[r];
      R.d1 = it.rowd[r];
      if (!act) continue;
      const float x1 = R.x1;
      int s, e;
      if (side == 0) {
        auto pa_pred = [&](float x2) { return x2 >= x1 && __fsub_rn(x2, x1) >= ta; };
        auto pb_pred = [&](float x2) { return x2 >= x1 && __fsub_rn(x2, x1) >= tb; };
        if (r == r_lo) {
          pa = bsearch_col(it.colx, 0, nj, pa_pred);
          pb = bsearch_col(it.colx, pa, nj, pb_pred);
        } else {
          while (pa < nj && !pa_pred(it.colx[pa])) ++pa;
          pb = max(pb, pa);
          while (pb < nj && !pb_pred(it.colx[pb])) ++pb;
        }
        s = pa;
        e = pb;
      } else {
        auto pa_pred = [&](float x2) { return x2 >= x1 || __fsub_rn(x1, x2) < ta; };
        auto pb_pred = [&](float x2) { return x2 >= x1 || __fsub_rn(x1, x2) < tb; };
        if (r == r_lo) {
          pb = bsearch_col(it.colx, 0, nj, pb_pred);
          pa = bsearch_col(it.colx, pb, nj, pa_pred);
        } else {
          while (pb < nj && !pb_pred(it.colx[pb])) ++pb;
          pa = max(pa, pb);
          while (pa < nj && !pa_pred(it.colx[pa])) ++pa;
        }
        s = pb;
        e = pa;
      }
      if (e > s) {
        n_eval += (unsigned long long)(e - s);
        R.wd1 = it.rowwd[r];
        R.w1 = (double)it.roww[r];
        R.hl1 = 0.5 * (double)it.rowl[r];
        if (COORD == kCart) {
          const float p = __fmul_rn(R.d1, R.d1);
          const float err = __fmaf_rn(R.d1, R.d1, -p);  // d1*d1 = p + err exactly
          R.A1 = __fmul_rn(R.d1, it.ap);
          R.dl1 = __fmul_rn(-err, A.inv1sqf);
        }
        do_run<COORD, MINPOS>(A, it, R, k, s, e, acc, n_recheck);
      }
    }
    if (act) {
      acc_flush<COORD>(A, it, k, acc.B, acc.s0);
      acc_flush<COORD>(A, it, k, acc.B + 1, acc.s1);
    }
  }
}

template <int COORD, bool MINPOS>
__global__ void __launch_bounds__(kRunWarps * 32, 1) run_kernel(PairArgs A) {
  const int lane = threadIdx.x & 31;
  unsigned long long n_eval = 0, n_recheck = 0, n_taken = 0;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(A.next_item, 1ull);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= A.n_items) break;
    RItem it;
    it.i = A.item_i[idx];
    it.j = A.item_j[idx];
    it.ni = A.npix[it.i];
    it.nj = A.npix[it.j];
    if (it.ni == 0 || it.nj == 0) continue;
    const float4 ri = A.range[it.i], rj = A.range[it.j];
    // z index constant over the item (else the pixel-pair kernel handles it)
    const float lsum_lo = __fadd_rn(ri.z, rj.z), lsum_hi = __fadd_rn(ri.w, rj.w);
    const double zlo = dmul(dsub(dmul(0.5, (double)lsum_lo), A.g.min2), A.g.invn2);
    const double zhi = dmul(dsub(dmul(0.5, (double)lsum_hi), A.g.min2), A.g.invn2);
    it.zb = zbin_of_sum(lsum_lo, A.g);
    const bool zconst = zlo > -1.0 && zhi < 2147483648.0 && it.zb == zbin_of_sum(lsum_hi, A.g);
    it.c = A.item_c[idx];
    if (!run_item(A, it.c, zconst)) continue;  // left to the pixel-pair kernel
    ++n_taken;
    it.cell = A.cell_idx[it.i];
    it.sep = (COORD == kObs) ? A.item_sep[idx] : 0u;
    const uint64_t oi = A.off[it.i] + (uint64_t)kPad * (it.i + 1);
    const uint64_t oj = A.off[it.j] + (uint64_t)kPad * (it.j + 1);
    it.rowd = A.dist_pad + oi;
    it.rowl = A.loglam_pad + oi;
    it.rowx = (COORD == kObs) ? it.rowl : it.rowd;
    it.rowwd = A.wd + A.off[it.i];
    it.roww = A.w + A.off[it.i];
    it.colx = (COORD == kObs) ? A.loglam_pad + oj : A.dist_pad + oj;
    it.pre = A.prefix + A.off[it.j] + it.j;
    it.col_min = (COORD == kObs) ? rj.z : rj.x;
    it.col_max = (COORD == kObs) ? rj.w : rj.y;
    const double a = 2.0 * dsub(1.0, it.c);
    it.ap = (float)(a * A.g.inv1 * A.g.inv1);
    sweep_item<COORD, MINPOS>(A, it, lane, n_eval, n_recheck);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_eval += __shfl_xor_sync(kFull, n_eval, o);
    n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  }
  if (lane == 0) {
    atomicAdd(&A.counters[0], n_eval);
    atomicAdd(&A.counters[1], n_recheck);
    atomicAdd(&A.counters[8], n_taken);
  }
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
