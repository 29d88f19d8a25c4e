// Stand-in for Healpix_cxx 3.30's healpix_map.h with what HealpixBins.h
// uses (HealpixBins.h:20-80): a RING-ordered map of order `order`
// (nside = 2^order), ang2pix, pix2ang, max_pixrad and query_disc_inclusive.
// Pixel numbering and centres follow the RING scheme of Gorski et al. 2005
// (ApJ 622, 759), restated here; Healpix_cxx itself is not in the reference.
//
// query_disc_inclusive returns every pixel whose centre is within
// radius + R of the query direction, R = kPixradBound * sqrt(4 pi / npix),
// a bound above the largest centre-to-boundary distance of any pixel (the
// oracle's tests measure the real maximum against it).  That is a superset
// of the pixels the disc touches, so the neighbours XiEstimator visits
// include every sightline within the disc, and its exact cos(theta) cut
// decides which pairs count: the result does not depend on the superset.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <exception>
#include <string>
#include <vector>

enum Healpix_Ordering_Scheme { RING, NEST };

struct pointing {
  double theta, phi;
  pointing() : theta(0), phi(0) {}
  pointing(double t, double p) : theta(t), phi(p) {}
};

class PlanckError : public std::exception {
 public:
  explicit PlanckError(std::string m) : m_(std::move(m)) {}
  const char* what() const noexcept override { return m_.c_str(); }

 private:
  std::string m_;
};

namespace tosref_healpix {
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kPixradBound = 1.5;

// RING pixel of direction (theta, phi): rings of constant z, pixels
// counted from phi = 0 eastwards, north polar cap first.  Longitude is
// measured in quarter turns, tt = phi * 2/pi reduced into [0, 4).  Within
// 0.01 rad of a pole the cap's ring distance is taken from sin(theta),
// which keeps the precision cos(theta) loses there.
inline int64_t ang2pix_ring(int64_t nside, double theta, double phi) {
  const double z = std::cos(theta), za = std::fabs(z);
  const bool near_pole = theta < 0.01 || theta > kPi - 0.01;
  double tt = phi * (2.0 / kPi);
  if (tt < 0 || tt >= 4.0) {
    tt = std::fmod(tt, 4.0);
    if (tt < 0) tt += 4.0;
    if (tt >= 4.0) tt = 0.0;
  }
  const int64_t ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
  if (za <= 2.0 / 3.0) {  // equatorial belt
    const double a = nside * (0.5 + tt), b = nside * z * 0.75;
    const int64_t jp = static_cast<int64_t>(a - b), jm = static_cast<int64_t>(a + b);
    const int64_t ring = nside + 1 + jp - jm;  // 1 .. 2 nside + 1 counted from z = 2/3
    const int64_t kshift = 1 - (ring & 1);
    const int64_t ip = ((jp + jm - nside + kshift + 1 + 8 * nside) / 2) % (4 * nside);
    return ncap + (ring - 1) * 4 * nside + ip;
  }
  const double tp = tt - std::floor(tt);
  const double dist = (za < 0.99 || !near_pole) ? nside * std::sqrt(3 * (1 - za))
                                                : nside * std::sin(theta) / std::sqrt((1 + za) / 3);
  const int64_t jp = static_cast<int64_t>(tp * dist), jm = static_cast<int64_t>((1.0 - tp) * dist);
  const int64_t ring = jp + jm + 1;  // 1 .. nside from the pole
  int64_t ip = static_cast<int64_t>(tt * ring);
  if (ip >= 4 * ring) ip -= 4 * ring;
  return z > 0 ? 2 * ring * (ring - 1) + ip : npix - 2 * ring * (ring + 1) + ip;
}

// Centre (theta, phi) of RING pixel p.
inline void pix2ang_ring(int64_t nside, int64_t p, double* theta, double* phi) {
  const int64_t ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
  const double fact = 1.0 / (3.0 * nside * nside);
  double z;
  if (p < ncap) {  // north cap: ring r holds 4r pixels
    int64_t r = static_cast<int64_t>(0.5 * (1 + std::sqrt(1.0 + 2.0 * p)));
    while (2 * r * (r - 1) > p) --r;
    while (2 * (r + 1) * r <= p) ++r;
    const int64_t k = p - 2 * r * (r - 1);
    z = 1 - r * r * fact;
    *phi = (k + 0.5) * 0.5 * kPi / r;
  } else if (p < npix - ncap) {  // belt: 4 nside pixels per ring, alternate rings shifted
    const int64_t q = p - ncap, r = q / (4 * nside) + nside, k = q % (4 * nside);
    const double shift = ((r + nside) & 1) ? 0.0 : 0.5;
    z = (2 * nside - r) * 2.0 / (3.0 * nside);
    *phi = (k + shift) * 0.5 * kPi / nside;
  } else {  // south cap, mirror of the north
    const int64_t q = npix - 1 - p;
    int64_t r = static_cast<int64_t>(0.5 * (1 + std::sqrt(1.0 + 2.0 * q)));
    while (2 * r * (r - 1) > q) --r;
    while (2 * (r + 1) * r <= q) ++r;
    const int64_t k = 4 * r - 1 - (q - 2 * r * (r - 1));
    z = -(1 - r * r * fact);
    *phi = (k + 0.5) * 0.5 * kPi / r;
  }
  *theta = std::acos(std::max(-1.0, std::min(1.0, z)));
}
}  // namespace tosref_healpix

template <class T>
class Healpix_Map {
 public:
  Healpix_Map() {}
  Healpix_Map(int order, Healpix_Ordering_Scheme scheme) : order_(order) {
    if (scheme != RING) throw PlanckError("only RING ordering is available");
    if (order < 0 || order > 13) throw PlanckError("order out of range");
    nside_ = int64_t(1) << order;
    const int64_t npix = 12 * nside_ * nside_;
    centres_.resize(3 * npix);
    for (int64_t p = 0; p < npix; ++p) {
      double th, ph;
      tosref_healpix::pix2ang_ring(nside_, p, &th, &ph);
      centres_[3 * p] = std::sin(th) * std::cos(ph);
      centres_[3 * p + 1] = std::sin(th) * std::sin(ph);
      centres_[3 * p + 2] = std::cos(th);
    }
  }
  int64_t Nside() const { return nside_; }
  int64_t Npix() const { return 12 * nside_ * nside_; }
  double max_pixrad() const { return tosref_healpix::kPixradBound * std::sqrt(4 * tosref_healpix::kPi / Npix()); }
  int ang2pix(const pointing& p) const {
    if (!(p.theta >= 0 && p.theta <= tosref_healpix::kPi)) throw PlanckError("invalid theta");
    return static_cast<int>(tosref_healpix::ang2pix_ring(nside_, p.theta, p.phi));
  }
  pointing pix2ang(int pix) const {
    pointing p;
    tosref_healpix::pix2ang_ring(nside_, pix, &p.theta, &p.phi);
    return p;
  }
  void query_disc_inclusive(const pointing& ptg, double radius, std::vector<int>& listpix, int /*fact*/ = 1) const {
    listpix.clear();
    const double reach = radius + max_pixrad();
    const double cmin = reach >= tosref_healpix::kPi ? -2.0 : std::cos(reach);
    const double x = std::sin(ptg.theta) * std::cos(ptg.phi), y = std::sin(ptg.theta) * std::sin(ptg.phi),
                 z = std::cos(ptg.theta);
    const int64_t npix = Npix();
    for (int64_t p = 0; p < npix; ++p) {
      const double c = x * centres_[3 * p] + y * centres_[3 * p + 1] + z * centres_[3 * p + 2];
      if (c >= cmin) listpix.push_back(static_cast<int>(p));
    }
  }

 private:
  int order_ = 0;
  int64_t nside_ = 1;
  std::vector<double> centres_;
};
