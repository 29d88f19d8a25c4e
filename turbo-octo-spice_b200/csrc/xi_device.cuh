// xi_device.cuh — device helpers shared by the pixel-pair kernel
// (xi_kernels.cu) and the run-sweep kernel (xi_runs.cu): FP32 approximations,
// fixed-point conversion, 128-bit accumulation, and the exact re-binning that
// follows the reference's FP64 expression order.
#pragma once

#include "xi_kernels.cuh"

namespace tos {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
enum { kPolar = TOS_POLAR, kCart = TOS_CARTESIAN, kObs = TOS_OBSERVING };

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Fixed-point image round(c * scale) of a contribution, |c*scale| < 2^51.
__device__ __forceinline__ long long to_fixed(double c, double scale) {
  return __double_as_longlong(__fma_rn(c, scale, kMagic52)) - kMagic52Bits;
}

// round(c * 2^F) for |c * 2^F| < 2^62, given sh = 2^(F-44): the high part is
// rounded first and the exact remainder carries the low 44 bits.
__device__ __forceinline__ long long to_fixed_wide(double c, double sh) {
  const double v = c * sh;
  const long long qh = __double_as_longlong(__dadd_rn(v, kMagic52)) - kMagic52Bits;
  const double rem = v - (double)qh;  // exact, |rem| <= 0.5
  return (qh << 44) + to_fixed(rem, 17592186044416.0 /* 2^44 */);
}

// Window word of field k, part p (0 = low).
__device__ __forceinline__ int wword(int k, int p) {
  return (k < kSigned) ? 3 * k + p : 3 * kSigned + 2 * (k - kSigned) + p;
}
constexpr int kWordCount = 3 * kSigned + 2 * (7 - kSigned);      // 17
constexpr int kWordContrib = kWordCount + 1;                     // 18

// Global reduction add with no returned value (red, not atom): nothing in
// the thread waits for it.
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Add a signed value v (|v| < 2^95) to one field's sums {lo, hi} in the
// carry-free format of kAccWords: lo += v mod 2^32, hi += floor(v / 2^32).
__device__ __forceinline__ void add_wide(unsigned long long* lo, unsigned long long* hi, __int128 v) {
  red_add(lo, (unsigned long long)v & 0xFFFFFFFFull);
  const long long h = (long long)(v >> 32);
  if (h != 0) red_add(hi, (unsigned long long)h);
}
__device__ __forceinline__ void add128(unsigned long long* lo, unsigned long long* hi, long long q) {
  add_wide(lo, hi, (__int128)q);
}

// ---- exact re-binning (reference expression order) returning the two axis
// indices; z is handled per item.  Mirrors ref_bin_* in tos_common.h.
__device__ __forceinline__ bool exact_cart(float d1, float d2, double c, const RefGrid& g,
                                           uint32_t* b0, uint32_t* b1) {
  const double r1_sq = (double)fmul(d1, d1);
  const double two_r1_cos12 = dmul((double)fmul(2.0f, d1), c);
  const double r_para = (double)fabsf(fsub(d1, d2));
  const uint32_t p = ref_u32(dmul(dsub(r_para, g.min0), g.inv0));
  if (p >= g.n0) return false;
  const double r_sq = dadd(r1_sq, dmul(dsub((double)d2, two_r1_cos12), (double)d2));
  const double x = fabs(dsub(r_sq, dmul(r_para, r_para)));
  const uint32_t q = ref_u32(dmul(dsub(dsqrt(x), g.min1), g.inv1));
  if (q >= g.n1) return false;
  *b0 = p;
  *b1 = q;
  return true;
}

__device__ __forceinline__ bool exact_polar(float d1, float d2, double c, const RefGrid& g,
                                            uint32_t* b0, uint32_t* b1) {
  const double r1_sq = (double)fmul(d1, d1);
  const double two_r1_cos12 = dmul((double)fmul(2.0f, d1), c);
  const double r_sq = dadd(r1_sq, dmul(dsub((double)d2, two_r1_cos12), (double)d2));
  const double r = dsqrt(r_sq);
  const uint32_t p = ref_u32(dmul(dsub(r, g.min0), g.inv0));
  if (p >= g.n0) return false;
  if (r == 0) return false;
  const double mu = ddiv((double)fabsf(fsub(d1, d2)), r);
  const uint32_t q = ref_u32(dmul(dsub(mu, g.min1), g.inv1));
  if (q >= g.n1) return false;
  *b0 = p;
  *b1 = q;
  return true;
}

__device__ __forceinline__ bool exact_obs(float l1, float l2, const RefGrid& g, uint32_t* b0) {
  const uint32_t p = ref_u32(dmul(dsub((double)fabsf(fsub(l1, l2)), g.min0), g.inv0));
  if (p >= g.n0) return false;
  *b0 = p;
  return true;
}

// Items of the run-sweep kernel when A.run_split is set: z index constant
// over the item and (Cartesian) 2(1 - cos theta) large enough for the
// reference's r_perp expression to grow with the column distance along every
// row.  Both kernels evaluate this same predicate.
__device__ __forceinline__ bool run_item(const PairArgs& A, double c, bool zconst) {
  return zconst && dmul(2.0, dsub(1.0, c)) >= A.run_amin;
}

// Run items whose sightlines are both contiguous on the common grid: the
// grid-sweep kernel's share when A.grid_split is set.
__device__ __forceinline__ bool grid_item(const PairArgs& A, uint32_t i, uint32_t j) {
  return A.grid_split && A.gfirst[i] != kNoGrid && A.gfirst[j] != kNoGrid;
}

__device__ __forceinline__ uint32_t zbin_of_sum(float lsum, const RefGrid& g) {
  return ref_u32(dmul(dsub(dmul(0.5, (double)lsum), g.min2), g.invn2));
}

// Items of the diagonal-sweep kernel when A.diag_split is set (Polar): the z
// index is constant over the item (from the z codes zlo, zhi of the smallest
// and largest loglam sums and their indices).  Both the diagonal-sweep and
// the pixel-pair kernel evaluate this same predicate.
__device__ __forceinline__ bool diag_item(const PairArgs& A, double zlo, double zhi, uint32_t zb_lo,
                                          uint32_t zb_hi) {
  return A.diag_split && zlo > -1.0 && zhi < 2147483648.0 && zb_lo == zb_hi;
}

// The kernel that takes item idx, from the predicates above as each kernel
// applies them (load_item and grid_item for the sweeps, the pixel-pair
// kernel's own test): one lane per item, so that a kernel can claim a batch
// of items and skip the others' without loading each one warp-wide.
enum ItemOwner { kOwnerNone = 0, kOwnerGrid, kOwnerRun, kOwnerDiag, kOwnerPair };
__device__ __forceinline__ int item_owner(const PairArgs& A, unsigned long long idx) {
  const uint32_t i = A.item_i[idx], j = A.item_j[idx];
  if (A.npix[i] == 0 || A.npix[j] == 0) return kOwnerNone;
  const float4 ri = A.range[i], rj = A.range[j];
  const float lsum_lo = __fadd_rn(ri.z, rj.z), lsum_hi = __fadd_rn(ri.w, rj.w);
  const double zlo = dmul(dsub(dmul(0.5, (double)lsum_lo), A.g.min2), A.g.invn2);
  const double zhi = dmul(dsub(dmul(0.5, (double)lsum_hi), A.g.min2), A.g.invn2);
  const uint32_t zb_lo = zbin_of_sum(lsum_lo, A.g), zb_hi = zbin_of_sum(lsum_hi, A.g);
  const bool zconst = zlo > -1.0 && zhi < 2147483648.0 && zb_lo == zb_hi;
  if (A.run_split && run_item(A, A.item_c[idx], zconst)) return grid_item(A, i, j) ? kOwnerGrid : kOwnerRun;
  if (diag_item(A, zlo, zhi, zb_lo, zb_hi)) return kOwnerDiag;
  return kOwnerPair;
}

// Items per claim of a kernel that takes few of the items (the run sweep and
// the pixel-pair kernel beside the grid or diagonal sweep): a warp claims 32
// with one atomic and keeps its own.
constexpr int kClaimItems = 32;

}  // namespace
}  // namespace tos
