// healpix.cc — RING-scheme ang2pix / pix2ang (Gorski et al. 2005).
//
// Geometry recap.  The sphere is split into 12*nside^2 equal-area pixels on
// 4*nside-1 iso-latitude rings.  Rings 1..nside-1 (north cap, z > 2/3) hold
// 4*i pixels; rings nside..3*nside (equatorial belt, |z| <= 2/3) hold
// 4*nside pixels each, alternately shifted by half a pixel; the south cap
// mirrors the north.  Pixels are numbered ring by ring from the north pole,
// eastwards from phi = 0 within a ring.
#include "healpix.h"

#include <cmath>

namespace tos {

namespace {
constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kTwoThirds = 2.0 / 3.0;
constexpr double kInvHalfPi = 0.6366197723675813430755350534900574;  // 2/pi

// v modulo m into [0, m).
inline double mod_positive(double v, double m) {
  if (v >= 0) return (v < m) ? v : std::fmod(v, m);
  double r = std::fmod(v, m) + m;
  return (r == m) ? 0.0 : r;
}

int64_t ring_index(int64_t nside, double z, double sin_theta, bool have_sin, double phi) {
  const double za = std::fabs(z);
  // longitude in units of quarter turns, in [0, 4)
  const double tt = mod_positive(phi * kInvHalfPi, 4.0);
  const int64_t npix = 12 * nside * nside;
  const int64_t ncap = 2 * nside * (nside - 1);  // pixels in the north cap
  if (za <= kTwoThirds) {
    // Equatorial belt: pixel edges are the lines z = 4/3 - 8 phi/(3 pi) (+/- k),
    // indexed by jp (ascending) and jm (descending).
    const int64_t nl4 = 4 * nside;
    const double t1 = nside * (0.5 + tt);
    const double t2 = nside * z * 0.75;
    const int64_t jp = (int64_t)(t1 - t2);
    const int64_t jm = (int64_t)(t1 + t2);
    const int64_t ring = nside + 1 + jp - jm;  // 1 .. 2 nside + 1, counted from z = 2/3
    const int64_t odd_shift = 1 - (ring & 1);
    int64_t ip = (jp + jm - nside + odd_shift + 1 + 2 * nl4) / 2;
    ip %= nl4;
    return ncap + (ring - 1) * nl4 + ip;
  }
  // Polar caps: distance from the pole in units where rings are equally spaced.
  const double tp = tt - (double)(int64_t)tt;
  const double dist = (za < 0.99 || !have_sin) ? nside * std::sqrt(3.0 * (1.0 - za))
                                               : nside * sin_theta / std::sqrt((1.0 + za) / 3.0);
  const int64_t jp = (int64_t)(tp * dist);
  const int64_t jm = (int64_t)((1.0 - tp) * dist);
  const int64_t ring = jp + jm + 1;  // ring counted from the nearest pole
  int64_t ip = (int64_t)(tt * (double)ring);
  if (ip >= 4 * ring) ip -= 4 * ring;  // wrap, as the published algorithm does
  return (z > 0) ? 2 * ring * (ring - 1) + ip : npix - 2 * ring * (ring + 1) + ip;
}
}  // namespace

int64_t healpix_ang2pix_ring(int64_t nside, double theta, double phi) {
  // Near the poles, cos(theta) loses the information sin(theta) keeps.
  if (theta < 0.01 || theta > kPi - 0.01)
    return ring_index(nside, std::cos(theta), std::sin(theta), true, phi);
  return ring_index(nside, std::cos(theta), 0.0, false, phi);
}

int64_t healpix_radec2pix(int64_t nside, double ra, double dec) {
  const double pi = std::atan(1.0) * 4;  // turbooctospice::pi (constants.h:9)
  return healpix_ang2pix_ring(nside, 0.5 * pi - dec, ra);
}

void healpix_pix2ang_ring(int64_t nside, int64_t pix, double* theta, double* phi) {
  const int64_t npix = 12 * nside * nside;
  const int64_t ncap = 2 * nside * (nside - 1);
  const double fact2 = 4.0 / (double)npix;
  if (pix < ncap) {  // north cap
    const int64_t ring = (int64_t)((1 + (int64_t)std::sqrt(1.0 + 2.0 * (double)pix)) / 2);
    int64_t r = ring;
    while (2 * r * (r - 1) > pix) --r;
    while (2 * (r + 1) * r <= pix) ++r;
    const int64_t iphi = pix + 1 - 2 * r * (r - 1);
    const double z = 1.0 - (double)(r * r) * fact2;
    *theta = std::acos(z);
    *phi = ((double)iphi - 0.5) * (kPi / 2.0) / (double)r;
  } else if (pix < npix - ncap) {  // equatorial belt
    const int64_t ip = pix - ncap;
    const int64_t nl4 = 4 * nside;
    const int64_t ring = ip / nl4 + nside;  // counted from the north pole
    const int64_t iphi = ip % nl4 + 1;
    const double fodd = ((ring + nside) & 1) ? 1.0 : 0.5;
    const double z = (double)(2 * nside - ring) * (2.0 / 3.0) / (double)nside;
    *theta = std::acos(z);
    *phi = ((double)iphi - fodd) * kPi / (2.0 * (double)nside);
  } else {  // south cap
    const int64_t ip = npix - pix;
    int64_t r = (int64_t)((1 + (int64_t)std::sqrt(2.0 * (double)ip - 1.0)) / 2);
    if (r < 1) r = 1;
    while (2 * r * (r - 1) >= ip) --r;
    while (2 * (r + 1) * r < ip) ++r;
    const int64_t iphi = 4 * r + 1 - (ip - 2 * r * (r - 1));
    const double z = -1.0 + (double)(r * r) * fact2;
    *theta = std::acos(z);
    *phi = ((double)iphi - 0.5) * (kPi / 2.0) / (double)r;
  }
}

}  // namespace tos
