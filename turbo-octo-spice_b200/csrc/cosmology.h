// cosmology.h — the pixel distance of h5healxi (h5healxi.cc:38-40, 196-203)
// as one host/device function, so that the host fill (tos_fill_distances)
// and the device fill of tos_catalog_create_dc give the same float for every
// pixel, bit for bit.
//
//   z = 10^(loglam - log10(1216)) - 1            (constants.h:10-11)
//   D = (c / 100 km/s/Mpc) * int_0^z dz' / E(z'),  E = sqrt(Om (1+z)^3 + 1 - Om)
//
// The integral is a table of D at z = k dz (cosmology.cc), evaluated between
// nodes by cubic Hermite interpolation with the exact derivative 1/E.  Every
// operation is one IEEE-rounded double operation (tos_common.h: no fused
// multiply-add on either side), and 10^x is computed here rather than by the
// platform's pow, whose rounding differs between libm and CUDA:
//   10^x = 2^k e^r,  t = x ln 10,  k = nearest integer to t / ln 2,
//   r = (t - k ln2_hi) - k ln2_lo  (|r| <= 0.35; ln 2 split so k ln2_hi is exact),
//   e^r by its Taylor series to the r^16 term in Horner form (remainder < 1e-19),
//   2^k exactly from the exponent bits.
// The result is within a few units in the last place of 10^x.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "tos_common.h"

namespace tos {

constexpr double kHubbleDistance = 2997.92458;  // c / (100 km/s/Mpc) in Mpc/h
constexpr double kLn10 = 2.302585092994045684;
constexpr double kLn2Hi = 0.693147180369123816490;   // ln 2 to 32 bits: k * kLn2Hi exact for |k| < 2^20
constexpr double kLn2Lo = 1.90821492927058770002e-10;  // ln 2 - kLn2Hi
constexpr double kInvLn2 = 1.44269504088896338700;

TOS_HD double pow2i(int k) {  // 2^k for |k| < 1000
  const uint64_t bits = (uint64_t)(k + 1023) << 52;
  double v;
#ifdef __CUDA_ARCH__
  v = __longlong_as_double((long long)bits);
#else
  std::memcpy(&v, &bits, 8);
#endif
  return v;
}

// 10^x for |x| < 300, the same bits on host and device.
TOS_HD double exp10_hd(double x) {
  const double t = dmul(x, kLn10);
  const double kd = floor(dadd(dmul(t, kInvLn2), 0.5));
  const int k = (int)kd;
  const double r = dsub(dsub(t, dmul(kd, kLn2Hi)), dmul(kd, kLn2Lo));
  double p = 1.0;
  for (int n = 16; n >= 1; --n) p = dadd(1.0, dmul(ddiv(r, (double)n), p));
  return dmul(p, pow2i(k));
}

// 1 / E(z) of flat LCDM.
TOS_HD double inv_e_hd(double om, double z) {
  const double a = dadd(1.0, z);
  return ddiv(1.0, dsqrt(dadd(dmul(dmul(dmul(om, a), a), a), dsub(1.0, om))));
}

// D_C(z) / (c / 100 km/s/Mpc) from the table d[k] = D_C(k dz) (n entries).
TOS_HD double dc_eval_hd(const double* d, size_t n, double om, double dz, double z) {
  const double u = ddiv(z, dz);
  size_t k = (size_t)u;
  if (k + 1 >= n) k = n - 2;
  const double s = dsub(u, (double)k);
  const double y0 = d[k], y1 = d[k + 1];
  const double m0 = dmul(inv_e_hd(om, dmul((double)k, dz)), dz);
  const double m1 = dmul(inv_e_hd(om, dmul((double)(k + 1), dz)), dz);
  const double s2 = dmul(s, s), s3 = dmul(s2, s);
  const double h00 = dadd(dsub(dmul(2.0, s3), dmul(3.0, s2)), 1.0);
  const double h10 = dadd(dsub(s3, dmul(2.0, s2)), s);
  const double h01 = dadd(dmul(-2.0, s3), dmul(3.0, s2));
  const double h11 = dsub(s3, s2);
  return dadd(dadd(dadd(dmul(h00, y0), dmul(h10, m0)), dmul(h01, y1)), dmul(h11, m1));
}

// The pixel redshift of a log10 wavelength (h5healxi.cc:38-40).
TOS_HD double pixel_z_hd(float loglam, double log_lya) { return dsub(exp10_hd(dsub((double)loglam, log_lya)), 1.0); }

// The pixel distance in Mpc/h, as stored (float).
TOS_HD float pixel_distance_hd(float loglam, double log_lya, const double* d, size_t n, double om, double dz) {
  return (float)dmul(kHubbleDistance, dc_eval_hd(d, n, om, dz, pixel_z_hd(loglam, log_lya)));
}

// Host side (cosmology.cc): log10(1216), and a copy of the D_C table for a
// matter density and largest redshift (the table tos_fill_distances uses).
double log_lya();
void dc_table(double om, double zmax, std::vector<double>* d, double* dz);

}  // namespace tos
