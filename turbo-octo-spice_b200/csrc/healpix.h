// healpix.h — HEALPix RING-scheme pixel index of a sky position.
//
// Replaces Healpix_cxx 3.30's Healpix_Base::ang2pix as HealpixBins calls it
// (HealpixBins.h:58-66, map built with scheme RING at HealpixBins.h:24).
// The formulas are the RING-scheme equations of Gorski et al. 2005,
// ApJ 622, 759 (section 4 and appendix), restated here; near the poles the
// polar-cap coordinate uses sin(theta) for accuracy as the HEALPix library
// does for |cos(theta)| > 0.99.
#pragma once

#include <cstdint>

namespace tos {

// Pixel index (RING) of the direction (theta, phi): theta colatitude in
// [0, pi], phi longitude in radians (any value; reduced modulo 2pi).
int64_t healpix_ang2pix_ring(int64_t nside, double theta, double phi);

// Sightline position (ra, dec) in radians to a RING pixel, as
// HealpixBins::ang2pix with radec2pnt: theta = pi/2 - dec, phi = ra
// (HealpixBins.h:58-72).
int64_t healpix_radec2pix(int64_t nside, double ra, double dec);

// Centre of a RING pixel as (theta, phi).
void healpix_pix2ang_ring(int64_t nside, int64_t pix, double* theta, double* phi);

}  // namespace tos
