// brute.cu — all-pairs isotropic xi(r) of points (x, y, z, delta, w): the
// computation of bruteGPU / histo_kernel (gpu/brute.cu:7-61, 63-225), redone
// for sm_100a.
//
// Differences from the reference design, all in service of exactness and
// throughput:
//  - points stay resident in HBM (no per-chunk host copies, brute.cu:155-193);
//  - every unordered pair i < j is visited once, along diagonals: a pair
//    (i, i + delta) lies on diagonal delta, a lane owns K consecutive
//    diagonals of a group of 32 K and walks them row by row (i = 0, 1, ...),
//    so the row's point is a broadcast load and the lane's K columns are a
//    register window that slides by one column per row.  For points on a
//    regular grid the separation vector of a diagonal stays the same along
//    whole runs of rows (until the column wraps to the next grid line), so
//    the bin of a diagonal changes only every few tens of rows;
//  - separations are binned in FP32 with an FP64 re-binning of pairs within
//    2^-K bins of an edge, so bins equal those of the FP64 separation
//    sqrt(dx^2+dy^2+dz^2) (the double-precision estimator of bucketxi.cc:79-98);
//  - sums are exact: while a diagonal stays in one bin the lane adds the
//    FP64 products w_i d_i w_j d_j and w_i w_j in registers; a run that ends
//    goes, rounded once to fixed point, into a per-warp shared-memory window
//    of 128-bit carry-free sums, which is added to the global sums after each
//    diagonal group.  Integer sums do not depend on the order of the adds, so
//    the result is the same for every launch shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "engine_internal.h"
#include "fixed128.cuh"

namespace tos {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBruteWarpsMax = 16;  // warps per CTA at most
constexpr int kBWin = 5;            // u64 words per bin of a window: dsum lo, hi, wsum lo, hi, count
constexpr int kBQueue = 64;         // closed runs a warp holds before it adds 32 of them
constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52
constexpr long long kMagicBits = 0x4338000000000000LL;

struct BruteArgs {
  const float4* pos;      // (x, y, z, w), n entries
  const double* wd;       // w*delta per point (exact product of the two floats)
  int n;
  int nbins;
  double min, max, spacing;
  float invf, offf, nbf, nbp1f;
  int k;
  float mag;
  int bits;
  double scale_hi[2];     // 2^(F - 44) of fields dsum, wsum: |run sum| * 2^F < 2^62
  const double* th;       // [nbins + 3] exact-index thresholds on r^2 (brute_thresholds)
  unsigned long long* acc;       // [nbins + 2][kBWin] 128-bit carry-free sums and counts
  unsigned long long* next;      // diagonal-group counter
  unsigned long long* counters;  // [0] FP64 re-binnings
};

// A run that ended: bin, pairs and its two FP64 sums.
struct BRun {
  uint32_t bin, m;
  double dsum, wsum;
};

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// round(c * 2^F) for |c * 2^F| < 2^62, given sh = 2^(F-44): the high part is
// rounded first and the exact remainder carries the low 44 bits.
__device__ __forceinline__ long long fixed_wide(double c, double sh) {
  const double v = c * sh;
  const long long qh = __double_as_longlong(__dadd_rn(v, kMagic)) - kMagicBits;
  const double rem = v - (double)qh;  // exact, |rem| <= 0.5
  const long long ql = __double_as_longlong(__fma_rn(rem, 17592186044416.0 /* 2^44 */, kMagic)) - kMagicBits;
  return (qh << 44) + ql;
}

// Histogram index of the FP64 separation, 0 below min, nbins+1 at or above
// max, else floor((r - min) / spacing) + 1 with r = sqrt(dx^2 + dy^2 + dz^2)
// in FP64 (gpu/brute.cu:40-48, bucketxi.cc:79-98).  The index is a
// non-decreasing function of the FP64 r^2, so th[b] (b = 1 .. nbins + 1) is
// the smallest r^2 whose index is at least b (brute_thresholds, with
// th[0] = -1 and th[nbins + 2] = +inf), and an index known to lie within one
// of `near` is decided by two comparisons of r^2.
__device__ __forceinline__ uint32_t exact_index(const BruteArgs& A, float4 a, float4 b, int near) {
  const double dx = dsub((double)a.x, (double)b.x), dy = dsub((double)a.y, (double)b.y),
               dz = dsub((double)a.z, (double)b.z);
  const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
  const int c = min(max(near, 0), A.nbins + 1);
  return (uint32_t)(c - 1 + (r2 >= A.th[c] ? 1 : 0) + (r2 >= A.th[c + 1] ? 1 : 0));
}

// Add the queued runs [first, first + cnt) to the warp window, one per lane.
__device__ __forceinline__ void brute_drain(const BruteArgs& A, unsigned long long* win, int S,
                                            const BRun* q, int first, int cnt, int lane) {
  __syncwarp();
  if (lane < cnt) {
    const BRun r = q[first + lane];
    const long long v0 = fixed_wide(r.dsum, A.scale_hi[0]);
    const long long v1 = fixed_wide(r.wsum, A.scale_hi[1]);
    atomicAdd(&win[0 * S + r.bin], (unsigned long long)v0 & 0xFFFFFFFFull);
    atomicAdd(&win[1 * S + r.bin], (unsigned long long)(v0 >> 32));
    atomicAdd(&win[2 * S + r.bin], (unsigned long long)v1 & 0xFFFFFFFFull);
    atomicAdd(&win[3 * S + r.bin], (unsigned long long)(v1 >> 32));
    atomicAdd(&win[4 * S + r.bin], (unsigned long long)r.m);
  }
  __syncwarp();
}

// Add the warp window to the global sums (carry-free: low 32 bits and the
// signed rest of each 128-bit window value) and clear it.
__device__ __forceinline__ void brute_flush(const BruteArgs& A, unsigned long long* win, int S, int lane) {
  __syncwarp();
  for (int b = lane; b < S; b += 32) {
    const unsigned long long cnt = win[4 * S + b];
    if (cnt == 0) continue;  // every run has at least one pair
    unsigned long long* g = A.acc + (size_t)b * kBWin;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const __int128 v = (__int128)(long long)win[(2 * f + 1) * S + b] * (__int128)4294967296ll +
                         (__int128)win[2 * f * S + b];
      atomicAdd(&g[2 * f], (unsigned long long)v & 0xFFFFFFFFull);
      const long long h = (long long)(v >> 32);
      if (h != 0) atomicAdd(&g[2 * f + 1], (unsigned long long)h);
      win[2 * f * S + b] = 0ull;
      win[(2 * f + 1) * S + b] = 0ull;
    }
    atomicAdd(&g[4], cnt);
    win[4 * S + b] = 0ull;
  }
  __syncwarp();
}

// Diagonal groups: group g holds diagonals 1 + g * 32K .. 1 + (g + 1) * 32K - 1;
// lane L owns 1 + g * 32K + K L + m, m = 0 .. K-1.  Longest diagonals first.
template <int K>
__global__ void __launch_bounds__(kBruteWarpsMax * 32) brute_kernel(BruteArgs A) {
  extern __shared__ unsigned long long bsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int S = A.nbins + 2;
  unsigned long long* win = bsm + (size_t)warp * kBWin * S;
  BRun* q = reinterpret_cast<BRun*>(bsm + (size_t)nw * kBWin * S) + warp * kBQueue;
  for (int k = lane; k < kBWin * S; k += 32) win[k] = 0ull;
  __syncwarp();
  const unsigned lt = (1u << lane) - 1u;
  const int span = 32 * K;
  const long long ngroups = ((long long)A.n - 1 + span - 1) / span;
  unsigned long long n_recheck = 0;
  for (;;) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(A.next, 1ull);
    g = __shfl_sync(kFull, g, 0);
    if (g >= (unsigned long long)ngroups) break;
    const int dg = 1 + (int)g * span;  // the group's first diagonal
    const int d0 = dg + K * lane;      // this lane's first diagonal
    const int t_end = A.n - dg;        // rows with a pair on the group's first diagonal
    uint32_t cur[K];
    int s0[K];
    double ds[K], ws[K];
    float4 cp[K];
    double cwd[K];
#pragma unroll
    for (int m = 0; m < K; ++m) {
      cur[m] = 0xFFFFFFFFu;
      s0[m] = 0;
      ds[m] = ws[m] = 0.0;
    }
    // columns of row 0: d0 + m (the newest, m = K - 1, is loaded in the loop)
#pragma unroll
    for (int m = 0; m + 1 < K; ++m) {
      cp[m] = make_float4(0.f, 0.f, 0.f, 0.f);
      cwd[m] = 0.0;
      if (d0 + m < A.n) {
        cp[m] = A.pos[d0 + m];
        cwd[m] = A.wd[d0 + m];
      }
    }
    int qn = 0;  // queued runs (the same in every lane)
    // the lane's newest column (t + d0 + K - 1) and the row, walked by pointer
    const float4* pj = A.pos + (d0 + K - 1);
    const double* wdj = A.wd + (d0 + K - 1);
    const int j_end = A.n - (d0 + K - 1);  // rows t < j_end have the newest column
#pragma unroll 1
    for (int t = 0; t < t_end; ++t) {
      if (t < j_end) {
        cp[K - 1] = pj[t];
        cwd[K - 1] = wdj[t];
      }
      const float4 pi = A.pos[t];
      const double wdi = A.wd[t], wi = (double)pi.w;
#pragma unroll
      for (int m = 0; m < K; ++m) {
        const bool in = t < j_end + (K - 1 - m);  // t + d0 + m < n
        const float dx = __fsub_rn(pi.x, cp[m].x), dy = __fsub_rn(pi.y, cp[m].y),
                    dz = __fsub_rn(pi.z, cp[m].z);
        const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
        const float tt = __fmaf_rn(sqrt_approx(r2), A.invf, A.offf);
        const int qq = __float_as_int(__fadd_rz(tt, A.mag)) - A.bits;
        int b = (qq >> A.k) + 1;
        b = (tt < 0.f) ? 0 : ((tt >= A.nbf) ? A.nbins + 1 : b);
        uint32_t key = in ? (uint32_t)b : 0xFFFFFFFFu;
        const bool recheck = in && (((qq + 1) & ((1 << A.k) - 1)) < 2) && (tt < A.nbp1f) && (tt > -1.f);
        if (__any_sync(kFull, recheck)) {
          if (recheck) {
            key = exact_index(A, pi, cp[m], b);
            ++n_recheck;
          }
        }
        const bool change = key != cur[m];
        const bool close = change && cur[m] != 0xFFFFFFFFu;
        const unsigned cm = __ballot_sync(kFull, close);
        if (cm) {
          if (close) q[qn + __popc(cm & lt)] = BRun{cur[m], (uint32_t)(t - s0[m]), ds[m], ws[m]};
          qn += __popc(cm);
          if (qn >= 32) {
            qn -= 32;
            brute_drain(A, win, S, q, qn, 32, lane);
          }
        }
        if (change) {
          cur[m] = key;
          s0[m] = t;
          ds[m] = 0.0;
          ws[m] = 0.0;
        }
        if (in) {
          ds[m] = __fma_rn(wdi, cwd[m], ds[m]);
          ws[m] = __fma_rn(wi, (double)cp[m].w, ws[m]);
        }
      }
#pragma unroll
      for (int m = 0; m + 1 < K; ++m) {
        cp[m] = cp[m + 1];
        cwd[m] = cwd[m + 1];
      }
    }
    // runs still open: a diagonal's last pair is at row n - 1 - delta, and
    // every row after it was out of range, which already closed the run
#pragma unroll
    for (int m = 0; m < K; ++m) {
      const bool close = cur[m] != 0xFFFFFFFFu;
      const unsigned cm = __ballot_sync(kFull, close);
      if (close) q[qn + __popc(cm & lt)] = BRun{cur[m], (uint32_t)(t_end - s0[m]), ds[m], ws[m]};
      qn += __popc(cm);
      if (qn >= 32) {
        qn -= 32;
        brute_drain(A, win, S, q, qn, 32, lane);
      }
    }
    brute_drain(A, win, S, q, 0, qn, lane);
    brute_flush(A, win, S, lane);
  }
  for (int o = 16; o > 0; o >>= 1) n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  if (lane == 0) atomicAdd(&A.counters[0], n_recheck);
}

__global__ void k_brute_prep(const float* pts, int n, float4* pos, double* wd) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float* p = pts + 5 * (size_t)k;
    pos[k] = make_float4(p[0], p[1], p[2], p[4]);
    wd[k] = (double)p[4] * (double)p[3];
  }
}

// 128-bit sums -> the caller's dsum, wsum (FP64) and counts.
__global__ void k_brute_finish(const unsigned long long* acc, int nb2, double inv0, double inv1, double* dsum,
                               double* wsum, uint64_t* counts) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb2; b += gridDim.x * blockDim.x) {
    const unsigned long long* g = acc + (size_t)b * kBWin;
    const __int128 v0 = (__int128)(long long)g[1] * (__int128)4294967296ll + (__int128)g[0];
    const __int128 v1 = (__int128)(long long)g[3] * (__int128)4294967296ll + (__int128)g[2];
    dsum[b] = i128_double(v0) * inv0;
    wsum[b] = i128_double(v1) * inv1;
    counts[b] = g[4];
  }
}

// The kernel's variants, by diagonals per lane.
struct BruteVariant {
  int k;
  void (*fn)(BruteArgs);
};
const BruteVariant kVariants[] = {{1, brute_kernel<1>}, {2, brute_kernel<2>}, {4, brute_kernel<4>}};

// Launch shape: per warp a window of kBWin words for each of the nbins + 2
// bins and a queue of kBQueue runs, so as many warps (up to `warps_max`) as
// the block's opt-in shared memory holds.  Fails only if not even one warp fits.
tos_status brute_shape(const tos_engine* e, int nbins, int warps_max, int* warps, size_t* smem) {
  const size_t per_warp = (size_t)kBWin * (nbins + 2) * 8 + (size_t)kBQueue * sizeof(BRun);
  const size_t fit = e->smem_optin / per_warp;
  if (fit < 1)
    return fail(TOS_ERR_UNSUPPORTED, "nbins too large for one warp's shared-memory window on this device");
  *warps = (int)std::min<size_t>((size_t)warps_max, fit);
  *smem = (size_t)*warps * per_warp;
  return TOS_OK;
}

// Fill the kernel arguments shared by both entry points (binning, FP32
// fast-path constants and the fixed-point scales from the bounds of |w d|
// and |w|: a run holds at most n - 1 pairs).
void brute_args(BruteArgs& A, int n, int nbins, double min, double max, double mwd, double mw) {
  A.n = n;
  A.nbins = nbins;
  A.min = min;
  A.max = max;
  A.spacing = (max - min) / nbins;
  A.invf = (float)(1.0 / A.spacing);
  A.offf = (float)(-min / A.spacing);
  A.nbf = (float)nbins;
  A.nbp1f = (float)nbins + 1.0f;
  int bl = 0;
  for (uint32_t v = (uint32_t)nbins + 2; v; v >>= 1) ++bl;
  A.k = std::max(0, std::min(13, 21 - bl));
  A.mag = std::ldexp(1.5f, 23 - A.k);
  std::memcpy(&A.bits, &A.mag, 4);
  const double per[2] = {mwd * mwd * (double)n, mw * mw * (double)n};
  for (int f = 0; f < 2; ++f) {
    int F = (int)std::floor(62.0 - std::log2(std::max(per[f], 1e-300)));
    F = std::max(-60, std::min(F, 200));
    A.scale_hi[f] = std::ldexp(1.0, F - 44);
  }
}

double brute_inv_scale(const BruteArgs& A, int f) { return 1.0 / (A.scale_hi[f] * 17592186044416.0); }

// The histogram index of an FP64 squared separation r2, computed as the
// reference's double-precision estimator does from r = sqrt(r2).
int brute_index_of_r2(double r2, double min, double max, double spacing, int nbins) {
  const double r = std::sqrt(r2);
  if (r < min) return 0;
  if (r >= max) return nbins + 1;
  double k = std::floor(tos::ddiv(tos::dsub(r, min), spacing));
  if (k > (double)(nbins - 1)) k = (double)(nbins - 1);
  return (int)k + 1;
}

// th[b], b = 1 .. nbins + 1: the smallest double r2 >= 0 whose index is at
// least b (bisection over the ordered bit patterns of non-negative doubles;
// the index is non-decreasing in r2), th[0] = -1, th[nbins + 2] = +inf.
// IEEE sqrt, subtraction and division round the same on the host and the
// device, so the device's comparisons reproduce the FP64 index exactly.
std::vector<double> brute_thresholds(double min, double max, int nbins) {
  std::vector<double> th((size_t)nbins + 3);
  th[0] = -1.0;
  th[(size_t)nbins + 2] = std::numeric_limits<double>::infinity();
  const double spacing = (max - min) / nbins;
  const uint64_t top = 0x7FF0000000000000ull;  // +inf
  for (int b = 1; b <= nbins + 1; ++b) {
    uint64_t lo = 0, hi = top;  // index(lo bits) < b <= index(hi bits) unless lo already reaches b
    double v;
    std::memcpy(&v, &lo, 8);
    if (brute_index_of_r2(v, min, max, spacing, nbins) >= b) {
      th[b] = 0.0;
      continue;
    }
    while (hi - lo > 1) {
      const uint64_t mid = lo + (hi - lo) / 2;
      std::memcpy(&v, &mid, 8);
      if (brute_index_of_r2(v, min, max, spacing, nbins) >= b) hi = mid; else lo = mid;
    }
    std::memcpy(&th[b], &hi, 8);
  }
  return th;
}

// Launch variant `vi` with up to `warps_max` warps per CTA, persistent (as
// many CTAs as fit on the SMs), between events ev[4] and ev[5].
tos_status brute_launch_shape(tos_engine* e, const BruteArgs& A, cudaStream_t st, int vi, int warps_max) {
  int warps = 0;
  size_t smem = 0;
  TOS_TRY(brute_shape(e, A.nbins, warps_max, &warps, &smem));
  const BruteVariant& v = kVariants[vi];
  TOS_CUDA_TRY(cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  TOS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, warps * 32, smem));
  TOS_CUDA_TRY(cudaEventRecord(e->ev[4], st));
  v.fn<<<e->num_sms * std::max(1, per_sm), warps * 32, smem, st>>>(A);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
  return TOS_OK;
}

// The default shape, or the one tos_brute_tune picked for this bin count.
constexpr int kBruteDefaultVariant = 0, kBruteDefaultWarps = 8;

tos_status brute_launch(tos_engine* e, const BruteArgs& A, cudaStream_t st) {
  int vi = kBruteDefaultVariant, warps_max = kBruteDefaultWarps;
  {
    std::lock_guard<std::mutex> lk(e->tune_mu);
    auto it = e->brute_tuned.find(A.nbins);
    if (it != e->brute_tuned.end()) {
      vi = it->second.first;
      warps_max = it->second.second;
    }
  }
  return brute_launch_shape(e, A, st, vi, warps_max);
}

}  // namespace
}  // namespace tos

using namespace tos;

extern "C" tos_status tos_brute_run(tos_engine* e, const float* points, size_t n_points, double min,
                                    double max, int nbins, double* dsum, double* wsum,
                                    uint64_t* counts, double* ms_kernel) {
  if (!e || !points || !dsum || !wsum || !counts) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_points < 2 || n_points > (1u << 24)) return fail(TOS_ERR_INVALID_ARG, "need 2 <= n <= 2^24 points");
  if (nbins <= 0 || nbins > 4096) return fail(TOS_ERR_INVALID_ARG, "nbins must be in [1, 4096]");
  if (!(max > min) || !std::isfinite(min) || !std::isfinite(max))
    return fail(TOS_ERR_INVALID_ARG, "need finite min < max");
  // bounds of |w*delta| and |w| for the fixed-point scale
  const int n = (int)n_points;
  double mwd = 1e-300, mw = 1e-300;
  for (int k = 0; k < n; ++k) {
    const float* p = points + 5 * (size_t)k;
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || !std::isfinite(p[3]) ||
        !std::isfinite(p[4]))
      return fail(TOS_ERR_INVALID_ARG, "points must be finite");
    mwd = std::max(mwd, std::fabs((double)p[4] * (double)p[3]));
    mw = std::max(mw, std::fabs((double)p[4]));
  }
  std::lock_guard<std::mutex> lock(e->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  const int nb2 = nbins + 2;
  cudaStream_t st = e->stream;
  DevBuf<float> d_pts;
  DevBuf<float4> d_pos;
  DevBuf<double> d_wd, d_out;
  DevBuf<unsigned long long> d_acc, d_misc;
  DevBuf<uint64_t> d_cnt;
  DevBuf<double> d_th;
  const std::vector<double> th = brute_thresholds(min, max, nbins);  // kept until the stream sync
  TOS_TRY(d_th.alloc(th.size()));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_th.p, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  TOS_TRY(d_pts.alloc((size_t)n * 5));
  TOS_TRY(d_pos.alloc(n));
  TOS_TRY(d_wd.alloc(n));
  TOS_TRY(d_acc.alloc((size_t)nb2 * kBWin));
  TOS_TRY(d_out.alloc((size_t)nb2 * 2));
  TOS_TRY(d_cnt.alloc(nb2));
  TOS_TRY(d_misc.alloc(4));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_pts.p, points, (size_t)n * 5 * sizeof(float),
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemsetAsync(d_acc.p, 0, (size_t)nb2 * kBWin * 8, st));
  TOS_CUDA_TRY(cudaMemsetAsync(d_misc.p, 0, 32, st));
  k_brute_prep<<<std::min(4096, (n + 255) / 256), 256, 0, st>>>(d_pts.p, n, d_pos.p, d_wd.p);
  TOS_CUDA_TRY(cudaGetLastError());
  BruteArgs A{};
  A.pos = d_pos.p;
  A.wd = d_wd.p;
  brute_args(A, n, nbins, min, max, mwd, mw);
  A.th = d_th.p;
  A.acc = d_acc.p;
  A.next = d_misc.p;
  A.counters = d_misc.p + 1;
  TOS_TRY(brute_launch(e, A, st));
  k_brute_finish<<<(nb2 + 127) / 128, 128, 0, st>>>(d_acc.p, nb2, brute_inv_scale(A, 0), brute_inv_scale(A, 1),
                                                   d_out.p, d_out.p + nb2, d_cnt.p);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaMemcpyAsync(dsum, d_out.p, (size_t)nb2 * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(wsum, d_out.p + nb2, (size_t)nb2 * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(counts, d_cnt.p, (size_t)nb2 * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  if (ms_kernel) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]);
    *ms_kernel = ms;
  }
  return TOS_OK;
}

// Autotuner of the brute-force kernel's launch shape: every variant (1, 2 or
// 4 diagonals per lane) with 4, 8 and 16 warps per CTA, timed on the first
// min(n, 131072) points, best of two timed launches after a warm-up.
extern "C" tos_status tos_brute_tune(tos_engine* e, const float* points, size_t n_points, double min,
                                     double max, int nbins, int* diagonals_per_lane, int* warps_per_cta) {
  if (!e || !points) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_points < 2 || n_points > (1u << 24)) return fail(TOS_ERR_INVALID_ARG, "need 2 <= n <= 2^24 points");
  if (nbins <= 0 || nbins > 4096) return fail(TOS_ERR_INVALID_ARG, "nbins must be in [1, 4096]");
  if (!(max > min) || !std::isfinite(min) || !std::isfinite(max))
    return fail(TOS_ERR_INVALID_ARG, "need finite min < max");
  const int n = (int)std::min<size_t>(n_points, 131072);
  double mwd = 1e-300, mw = 1e-300;
  for (int k = 0; k < n; ++k) {
    const float* p = points + 5 * (size_t)k;
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || !std::isfinite(p[3]) ||
        !std::isfinite(p[4]))
      return fail(TOS_ERR_INVALID_ARG, "points must be finite");
    mwd = std::max(mwd, std::fabs((double)p[4] * (double)p[3]));
    mw = std::max(mw, std::fabs((double)p[4]));
  }
  std::lock_guard<std::mutex> lock(e->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  const int nb2 = nbins + 2;
  cudaStream_t st = e->stream;
  DevBuf<float> d_pts;
  DevBuf<float4> d_pos;
  DevBuf<double> d_wd, d_th;
  DevBuf<unsigned long long> d_acc, d_misc;
  const std::vector<double> th = brute_thresholds(min, max, nbins);  // kept until the stream sync
  TOS_TRY(d_th.alloc(th.size()));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_th.p, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  TOS_TRY(d_pts.alloc((size_t)n * 5));
  TOS_TRY(d_pos.alloc(n));
  TOS_TRY(d_wd.alloc(n));
  TOS_TRY(d_acc.alloc((size_t)nb2 * kBWin));
  TOS_TRY(d_misc.alloc(4));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_pts.p, points, (size_t)n * 5 * sizeof(float), cudaMemcpyHostToDevice, st));
  k_brute_prep<<<std::min(4096, (n + 255) / 256), 256, 0, st>>>(d_pts.p, n, d_pos.p, d_wd.p);
  TOS_CUDA_TRY(cudaGetLastError());
  BruteArgs A{};
  A.pos = d_pos.p;
  A.wd = d_wd.p;
  brute_args(A, n, nbins, min, max, mwd, mw);
  A.th = d_th.p;
  A.acc = d_acc.p;
  A.next = d_misc.p;
  A.counters = d_misc.p + 1;
  const int warp_opts[3] = {4, 8, 16};
  float best = 0.f;
  int best_v = kBruteDefaultVariant, best_w = kBruteDefaultWarps;
  for (int vi = 0; vi < (int)(sizeof(kVariants) / sizeof(kVariants[0])); ++vi) {
    for (int wo : warp_opts) {
      float t_min = 0.f;
      for (int rep = 0; rep < 3; ++rep) {
        TOS_CUDA_TRY(cudaMemsetAsync(d_acc.p, 0, (size_t)nb2 * kBWin * 8, st));
        TOS_CUDA_TRY(cudaMemsetAsync(d_misc.p, 0, 32, st));
        TOS_TRY(brute_launch_shape(e, A, st, vi, wo));
        TOS_CUDA_TRY(cudaEventSynchronize(e->ev[5]));
        float ms = 0.f;
        TOS_CUDA_TRY(cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]));
        if (rep > 0 && (rep == 1 || ms < t_min)) t_min = ms;
      }
      if (best == 0.f || t_min < best) {
        best = t_min;
        best_v = vi;
        best_w = wo;
      }
    }
  }
  {
    std::lock_guard<std::mutex> lk(e->tune_mu);
    e->brute_tuned[nbins] = std::make_pair(best_v, best_w);
  }
  if (diagonals_per_lane) *diagonals_per_lane = kVariants[best_v].k;
  if (warps_per_cta) *warps_per_cta = best_w;
  return TOS_OK;
}

// ============================================================================
// Allocation-free variant of tos_brute_run.
//
// Some callers cannot allocate device memory while they count pairs: code
// that manages every byte of the GPU through its own pool, code that runs
// where a cudaMalloc would synchronise the device or is not allowed, or
// service loops that must not touch the allocator at all.  tos_brute_run allocates its
// scratch on every call; tos_brute_run_noalloc takes its inputs and outputs
// in device memory and keeps all scratch in one statically sized device
// array that the library reserves on every GPU that loads it, until exit.
// ============================================================================

namespace tos {
namespace {

constexpr size_t kNoAllocMaxPoints = size_t(1) << 18;  // 262,144 points (a 64^3 grid)
constexpr int kNoAllocMaxBins = 4096;

constexpr size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
// scratch layout (byte offsets, each 256-byte aligned)
constexpr size_t kNaPos = 0;                                                  // float4[n]
constexpr size_t kNaWd = kNaPos + round256(16 * kNoAllocMaxPoints);           // double[n]
constexpr size_t kNaAcc = kNaWd + round256(8 * kNoAllocMaxPoints);            // u64[nbins + 2][kBWin]
constexpr size_t kNaTh = kNaAcc + round256(8 * kBWin * (kNoAllocMaxBins + 2));  // double[nbins + 3]
constexpr size_t kNaMisc = kNaTh + round256(8 * (kNoAllocMaxBins + 3));         // u64[8]
constexpr size_t kNoAllocBytes = kNaMisc + 256;                               // ~6.5 MB

// The scratch.  Host code must not pass this name to a kernel: on the host
// it stands for a host-side shadow, not for the device memory; the device
// address comes from cudaGetSymbolAddress (noalloc_scratch below).
static __device__ __align__(256) unsigned char g_brute_scratch[kNoAllocBytes];

// max |w * delta| and max |w| (as ordered bit patterns of non-negative
// doubles) and a flag for non-finite coordinates, weights or deltas
__global__ void k_brute_bounds(const float* pts, int n, unsigned long long* maxbits,
                               unsigned long long* bad) {
  double mwd = 0, mw = 0;
  bool nonfinite = false;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float* p = pts + 5 * (size_t)k;
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || !isfinite(p[3]) || !isfinite(p[4]))
      nonfinite = true;
    mwd = fmax(mwd, fabs((double)p[4] * (double)p[3]));
    mw = fmax(mw, fabs((double)p[4]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mwd = fmax(mwd, __shfl_xor_sync(kFull, mwd, o));
    mw = fmax(mw, __shfl_xor_sync(kFull, mw, o));
  }
  nonfinite = __any_sync(kFull, nonfinite);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(mwd));
    atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(mw));
    if (nonfinite) atomicOr(bad, 1ull);
  }
}

// Device address of g_brute_scratch on `device` (current): looked up once per
// device; the lookup may load the module on that device.
tos_status noalloc_scratch(int device, unsigned char** out) {
  static std::mutex mu;
  static std::vector<unsigned char*> addr;
  std::lock_guard<std::mutex> lock(mu);
  if ((size_t)device >= addr.size()) addr.resize(device + 1, nullptr);
  if (!addr[device]) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_brute_scratch);
    if (err != cudaSuccess || !p)
      return fail(TOS_ERR_CUDA, std::string("cudaGetSymbolAddress of the brute scratch: ") +
                                    cudaGetErrorString(err));
    addr[device] = (unsigned char*)p;
  }
  *out = addr[device];
  return TOS_OK;
}

}  // namespace
}  // namespace tos

extern "C" tos_status tos_brute_run_noalloc(tos_engine* e, const float* d_points, size_t n_points,
                                            double min, double max, int nbins, double* d_dsum,
                                            double* d_wsum, uint64_t* d_counts, double* ms_kernel) {
  if (!e || !d_points || !d_dsum || !d_wsum || !d_counts) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_points < 2) return fail(TOS_ERR_INVALID_ARG, "need at least 2 points");
  if (n_points > kNoAllocMaxPoints)
    return fail(TOS_ERR_INVALID_ARG, "tos_brute_run_noalloc takes at most " +
                                         std::to_string(kNoAllocMaxPoints) + " points (got " +
                                         std::to_string(n_points) + "); use tos_brute_run");
  if (nbins <= 0 || nbins > kNoAllocMaxBins)
    return fail(TOS_ERR_INVALID_ARG, "nbins must be in [1, " + std::to_string(kNoAllocMaxBins) + "]");
  if (!(max > min) || !std::isfinite(min) || !std::isfinite(max))
    return fail(TOS_ERR_INVALID_ARG, "need finite min < max");
  std::lock_guard<std::mutex> lock(e->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  unsigned char* S = nullptr;
  TOS_TRY(noalloc_scratch(e->device, &S));
  const int n = (int)n_points;
  const int nb2 = nbins + 2;
  cudaStream_t st = e->stream;
  float4* pos = (float4*)(S + kNaPos);
  double* wd = (double*)(S + kNaWd);
  unsigned long long* acc = (unsigned long long*)(S + kNaAcc);
  double* thr = (double*)(S + kNaTh);
  unsigned long long* misc = (unsigned long long*)(S + kNaMisc);  // [0] group counter [1] rechecks
                                                                   // [2,3] bounds [4] non-finite
  const std::vector<double> th = brute_thresholds(min, max, nbins);  // kept until the stream sync
  TOS_CUDA_TRY(cudaMemcpyAsync(thr, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  // the scratch keeps the previous call's contents: clear what accumulates
  TOS_CUDA_TRY(cudaMemsetAsync(acc, 0, (size_t)nb2 * kBWin * sizeof(unsigned long long), st));
  TOS_CUDA_TRY(cudaMemsetAsync(misc, 0, 8 * sizeof(unsigned long long), st));
  k_brute_bounds<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(d_points, n, misc + 2, misc + 4);
  k_brute_prep<<<std::min(4096, (n + 255) / 256), 256, 0, st>>>(d_points, n, pos, wd);
  TOS_CUDA_TRY(cudaGetLastError());
  unsigned long long hb[3] = {0, 0, 0};
  TOS_CUDA_TRY(cudaMemcpyAsync(hb, misc + 2, sizeof(hb), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  if (hb[2]) return fail(TOS_ERR_INVALID_ARG, "points must be finite");
  double mwd, mw;
  std::memcpy(&mwd, &hb[0], 8);
  std::memcpy(&mw, &hb[1], 8);
  mwd = std::max(mwd, 1e-300);
  mw = std::max(mw, 1e-300);
  // the same kernel and arguments as tos_brute_run, pointing into the scratch
  BruteArgs A{};
  A.pos = pos;
  A.wd = wd;
  brute_args(A, n, nbins, min, max, mwd, mw);
  A.th = thr;
  A.acc = acc;
  A.next = misc;
  A.counters = misc + 1;
  TOS_TRY(brute_launch(e, A, st));
  k_brute_finish<<<(nb2 + 127) / 128, 128, 0, st>>>(acc, nb2, brute_inv_scale(A, 0), brute_inv_scale(A, 1),
                                                   d_dsum, d_wsum, d_counts);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  if (ms_kernel) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]);
    *ms_kernel = ms;
  }
  return TOS_OK;
}
