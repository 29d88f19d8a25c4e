// tos_common.h — types and exact reference arithmetic shared by the host code
// and the CUDA kernels of the pair-counting engine.
//
// The "ref_*" functions reproduce, operation by operation, the double/float
// arithmetic of XiEstimator::accumulate_pixel_pairs (XiEstimator.cc:161-296)
// as C++ evaluates it without contraction: every double op is rounded once
// (no FMA), float*float and float+float stay float, and the conversion
// static_cast<unsigned>(double) follows the x86-64 code the reference build
// emits (cvttsd2si to a 64-bit register, low 32 bits kept).  On the device the
// explicit __d*_rn / __f*_rn intrinsics forbid contraction; host code that
// includes this header is compiled with -ffp-contract=off.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/tos_b200.h"

#ifdef __CUDACC__
#define TOS_HD __host__ __device__ __forceinline__
#else
#define TOS_HD inline
#endif

namespace tos {

// Padding of the per-sightline float arrays (distance, loglam): 32 sentinel
// entries before every sightline and after the last one, so a warp that
// reads a sightline at offsets [-32, N+32) never leaves the allocation.
constexpr int kPad = 32;
// Sentinel value of padded entries: far beyond any binnable separation, and
// finite so that differences of sentinels never produce NaN.
constexpr float kSentinel = 1.0e30f;

// A pixel's distance, weight and w*delta in one 16-byte load (the padded
// layout of the distance array; padding entries have distance kSentinel and
// zero weights).
struct alignas(16) PixPack {
  float d, w;
  double wd;
};

// ---- exact scalar ops -------------------------------------------------------
#ifdef __CUDA_ARCH__
TOS_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
TOS_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
TOS_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
TOS_HD double dsqrt(double a) { return __dsqrt_rn(a); }
TOS_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
TOS_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
TOS_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
TOS_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
#else
TOS_HD double dmul(double a, double b) { return a * b; }
TOS_HD double dadd(double a, double b) { return a + b; }
TOS_HD double dsub(double a, double b) { return a - b; }
TOS_HD double dsqrt(double a) { return std::sqrt(a); }
TOS_HD double ddiv(double a, double b) { return a / b; }
TOS_HD float fmul(float a, float b) { return a * b; }
TOS_HD float fadd(float a, float b) { return a + b; }
TOS_HD float fsub(float a, float b) { return a - b; }
#endif

// static_cast<unsigned>(x) as compiled for x86-64 (cvttsd2si r64, keep low 32
// bits): truncation toward zero; NaN and |x| >= 2^63 give the "integer
// indefinite" 0x8000000000000000, whose low 32 bits are 0.
TOS_HD uint32_t ref_u32(double x) {
  if (!(x > -9223372036854775808.0 && x < 9223372036854775808.0)) return 0u;
  return (uint32_t)(int64_t)x;
}

// ---- grid constants exactly as accumulate_pixel_pairs reads them -----------
// axis k: min = getAxisMin(k), inv = 1.0/getAxisBinWidth(k), n = getAxisNBins(k);
// the third axis is scaled by 1.0/getAxisNBins (XiEstimator.cc:174, 232, 268).
struct RefGrid {
  double min0, inv0, min1, inv1, min2, invn2;
  uint32_t n0, n1, n2, ntotal;
};

// Axis bin width as likely's uniform binning defines it: (max - min) / n.
inline double axis_width(const tos_axis& a) { return (a.max - a.min) / (double)a.nbins; }
// High edge of the last bin: min + n * width (AbsTwoPointGrid.cc:8-15).
inline double axis_high(const tos_axis& a) { return a.min + (double)a.nbins * axis_width(a); }

inline RefGrid make_ref_grid(const tos_grid& g) {
  RefGrid r;
  r.min0 = g.axis[0].min;
  r.inv0 = 1.0 / axis_width(g.axis[0]);
  r.min1 = g.axis[1].min;
  r.inv1 = 1.0 / axis_width(g.axis[1]);
  r.min2 = g.axis[2].min;
  r.invn2 = 1.0 / (double)g.axis[2].nbins;
  r.n0 = (uint32_t)g.axis[0].nbins;
  r.n1 = (uint32_t)g.axis[1].nbins;
  r.n2 = (uint32_t)g.axis[2].nbins;
  r.ntotal = r.n0 * r.n1 * r.n2;
  return r;
}

// z index of a pixel pair: 0.5*(float sum of loglams) (XiEstimator.cc:198-201,
// 251-253, 285-287).  No bounds check, as in the reference.
TOS_HD uint32_t ref_zbin(float l1, float l2, const RefGrid& g) {
  double lz = dmul(0.5, (double)fadd(l1, l2));
  return ref_u32(dmul(dsub(lz, g.min2), g.invn2));
}

// Cartesian branch, XiEstimator.cc:236-258.  Returns false when the pair is
// skipped; *idx is the unsigned (possibly out-of-grid) flat index.
TOS_HD bool ref_bin_cartesian(float d1, float l1, float d2, float l2, double c, const RefGrid& g,
                              uint32_t* idx) {
  const double r1_sq = (double)fmul(d1, d1);              // float product, then widened
  const double two_r1_cos12 = dmul((double)fmul(2.0f, d1), c);
  const double r_para = (double)fabsf(fsub(d1, d2));
  uint32_t b = ref_u32(dmul(dsub(r_para, g.min0), g.inv0));
  if (b >= g.n0) return false;
  const double r_sq = dadd(r1_sq, dmul(dsub((double)d2, two_r1_cos12), (double)d2));
  const double x = fabs(dsub(r_sq, dmul(r_para, r_para)));
  const uint32_t bp = ref_u32(dmul(dsub(dsqrt(x), g.min1), g.inv1));
  if (bp >= g.n1) return false;
  b = bp + b * g.n1;
  *idx = ref_zbin(l1, l2, g) + b * g.n2;
  return true;
}

// Polar branch, XiEstimator.cc:178-223.
TOS_HD bool ref_bin_polar(float d1, float l1, float d2, float l2, double c, const RefGrid& g,
                          uint32_t* idx) {
  const double r1_sq = (double)fmul(d1, d1);
  const double two_r1_cos12 = dmul((double)fmul(2.0f, d1), c);
  const double r_sq = dadd(r1_sq, dmul(dsub((double)d2, two_r1_cos12), (double)d2));
  const double r = dsqrt(r_sq);
  uint32_t b = ref_u32(dmul(dsub(r, g.min0), g.inv0));
  if (b >= g.n0) return false;
  if (r == 0) return false;
  const double mu = ddiv((double)fabsf(fsub(d1, d2)), r);
  const uint32_t mb = ref_u32(dmul(dsub(mu, g.min1), g.inv1));
  if (mb >= g.n1) return false;
  b = mb + b * g.n1;
  *idx = ref_zbin(l1, l2, g) + b * g.n2;
  return true;
}

// Observing (QuasarGrid) branch, XiEstimator.cc:274-291; sep_bin is the
// per-sightline-pair theta index of XiEstimator.cc:273 (unchecked).
TOS_HD bool ref_bin_observing(float l1, float l2, uint32_t sep_bin, const RefGrid& g,
                              uint32_t* idx) {
  uint32_t b = ref_u32(dmul(dsub((double)fabsf(fsub(l1, l2)), g.min0), g.inv0));
  if (b >= g.n0) return false;
  b = sep_bin + b * g.n1;
  *idx = ref_zbin(l1, l2, g) + b * g.n2;
  return true;
}

// cos(theta_ij) as SkyObject::angularSeparation (types.h:37-39), from the
// cached sin/cos of each sightline: sd*sd' + (cd*cd')*(sr*sr' + cr*cr').
struct SkyTrig {
  double sin_dec, cos_dec, sin_ra, cos_ra;
};
TOS_HD double ref_cos_sep(const SkyTrig& a, const SkyTrig& b) {
  return dadd(dmul(a.sin_dec, b.sin_dec),
              dmul(dmul(a.cos_dec, b.cos_dec),
                   dadd(dmul(a.sin_ra, b.sin_ra), dmul(a.cos_ra, b.cos_ra))));
}

}  // namespace tos
