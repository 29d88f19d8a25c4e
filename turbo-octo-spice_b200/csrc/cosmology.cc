// cosmology.cc — flat LCDM line-of-sight comoving distance in Mpc/h (host
// side: the table, tos_comoving_distance, tos_fill_distances; the per-pixel
// arithmetic is cosmology.h's, shared with the device fill).
//
// Replaces cosmo::LambdaCdmUniverse::getLineOfSightComovingDistance and the
// loglam -> distance loop of h5healxi (h5healxi.cc:38-40, 123-131, 196-203):
//   D_C(z) = (c / 100 km/s/Mpc) * int_0^z dz' / E(z'),
//   E(z) = sqrt(Om (1+z)^3 + (1 - Om)).
// The integral is tabulated once per Omega_m on a uniform z grid with
// 16-point Gauss-Legendre panels (error far below 1e-14 relative), and
// evaluated between nodes by cubic Hermite interpolation using the exact
// derivative 1/E at the nodes.
#include "cosmology.h"

#include <cmath>
#include <mutex>
#include <vector>

#include "../../include/tos_b200.h"

namespace {

// 16-point Gauss-Legendre nodes/weights on [-1, 1] (positive half).
constexpr double kGLx[8] = {0.0950125098376374, 0.2816035507792589, 0.4580167776572274,
                            0.6178762444026438, 0.7554044083550030, 0.8656312023878318,
                            0.9445750230732326, 0.9894009349916499};
constexpr double kGLw[8] = {0.1894506104550685, 0.1826034150449236, 0.1691565193950025,
                            0.1495959888165767, 0.1246289712555339, 0.0951585116824928,
                            0.0622535239386479, 0.0271524594117541};

struct Table {
  double om = -1;
  double dz = 1e-3;
  std::vector<double> d;  // D_C at z = k*dz, in units of c / (100 km/s/Mpc)
};

double panel(double om, double z0, double z1) {
  const double h = 0.5 * (z1 - z0), m = 0.5 * (z1 + z0);
  double s = 0;
  for (int k = 0; k < 8; ++k)
    s += kGLw[k] * (tos::inv_e_hd(om, m - h * kGLx[k]) + tos::inv_e_hd(om, m + h * kGLx[k]));
  return s * h;
}

std::mutex g_mu;
Table g_table;

// Caller holds g_mu.
const Table& table_for(double om, double zmax) {
  const size_t need = (size_t)std::ceil(zmax / g_table.dz) + 2;
  if (g_table.om != om || g_table.d.size() < need) {
    Table t;
    t.om = om;
    const size_t n = std::max<size_t>(need, 8192);
    t.d.resize(n);
    t.d[0] = 0;
    for (size_t k = 1; k < n; ++k)
      t.d[k] = t.d[k - 1] + panel(om, (k - 1) * t.dz, k * t.dz);
    g_table = std::move(t);
  }
  return g_table;
}

}  // namespace

namespace tos {

double log_lya() { return std::log10(1216.0); }  // turbooctospice::logLyA (constants.h:7-8)

void dc_table(double om, double zmax, std::vector<double>* d, double* dz) {
  std::lock_guard<std::mutex> lock(g_mu);
  const Table& t = table_for(om, zmax);
  *d = t.d;
  *dz = t.dz;
}

}  // namespace tos

extern "C" tos_status tos_comoving_distance(double omega_matter, const double* z, size_t n,
                                            double* out) {
  if ((n && (!z || !out)) || !(omega_matter > 0 && omega_matter <= 1)) return TOS_ERR_INVALID_ARG;
  double zmax = 0;
  for (size_t k = 0; k < n; ++k) {
    if (!(z[k] >= 0) || !std::isfinite(z[k])) return TOS_ERR_INVALID_ARG;
    zmax = std::max(zmax, z[k]);
  }
  std::lock_guard<std::mutex> lock(g_mu);
  const Table& t = table_for(omega_matter, zmax);
  for (size_t k = 0; k < n; ++k)
    out[k] = tos::dmul(tos::kHubbleDistance, tos::dc_eval_hd(t.d.data(), t.d.size(), t.om, t.dz, z[k]));
  return TOS_OK;
}

extern "C" tos_status tos_fill_distances(double omega_matter, tos_pixel* px, size_t n) {
  const double lya = tos::log_lya();
  if ((n && !px) || !(omega_matter > 0 && omega_matter <= 1)) return TOS_ERR_INVALID_ARG;
  double zmax = 0;
  for (size_t k = 0; k < n; ++k) {
    const double z = tos::pixel_z_hd(px[k].loglam, lya);  // h5healxi.cc:38-40
    if (!(z >= 0) || !std::isfinite(z)) return TOS_ERR_INVALID_ARG;
    zmax = std::max(zmax, z);
  }
  std::lock_guard<std::mutex> lock(g_mu);
  const Table& t = table_for(omega_matter, zmax);
  for (size_t k = 0; k < n; ++k)
    px[k].distance = tos::pixel_distance_hd(px[k].loglam, lya, t.d.data(), t.d.size(), t.om, t.dz);
  return TOS_OK;
}
