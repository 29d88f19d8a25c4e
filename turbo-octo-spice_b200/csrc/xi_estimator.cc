// xi_estimator.cc — XiEstimator facade (see xi_estimator.h).
#include "xi_estimator.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>

namespace tos {

namespace {
// boost::lexical_cast<std::string>(double) prints the shortest form with 17
// significant digits; for integers it prints plain decimals.
std::string lexical(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.17g", v);
  return buf;
}
std::string lexical(long long v) { return std::to_string(v); }

void check(tos_status s) {
  if (s != TOS_OK) throw RuntimeError(std::string("tos_b200: ") + tos_last_error());
}
}  // namespace

Axis Axis::parse(const std::string& spec) {
  // "[min:max]*n"
  Axis a;
  double lo, hi;
  int n;
  char tail;
  if (std::sscanf(spec.c_str(), " [%lf:%lf]*%d %c", &lo, &hi, &n, &tail) != 3 || n <= 0 || !(hi > lo))
    throw RuntimeError("bad binning specification: " + spec);
  a.min = lo;
  a.max = hi;
  a.nbins = n;
  return a;
}

TwoPointGrid::TwoPointGrid(tos_coord_type type, const Axis& a1, const Axis& a2, const Axis& a3) {
  g_.type = type;
  g_.reserved = 0;
  const Axis ax[3] = {a1, a2, a3};
  for (int k = 0; k < 3; ++k) {
    g_.axis[k].min = ax[k].min;
    g_.axis[k].max = ax[k].max;
    g_.axis[k].nbins = ax[k].nbins;
    g_.axis[k].reserved = 0;
  }
  if (tos_grid_num_bins(&g_) == 0) throw RuntimeError(std::string("invalid grid: ") + tos_last_error());
}

int TwoPointGrid::getNBinsTotal() const { return (int)tos_grid_num_bins(&g_); }

double TwoPointGrid::getAxisBinWidth(int axis) const {
  const tos_axis& a = g_.axis[axis];
  return (a.max - a.min) / (double)a.nbins;
}

double TwoPointGrid::getAxisMax(int axis) const {
  const tos_axis& a = g_.axis[axis];
  return a.min + (double)a.nbins * getAxisBinWidth(axis);
}

void TwoPointGrid::getBinCenters(int index, std::vector<double>& centers) const {
  // axis 0 varies slowest, axis 2 fastest: index = (i0*n1 + i1)*n2 + i2
  centers.resize(3);
  int rem = index;
  const int n2 = g_.axis[2].nbins, n1 = g_.axis[1].nbins;
  const int i2 = rem % n2;
  rem /= n2;
  const int i1 = rem % n1;
  const int i0 = rem / n1;
  const int idx[3] = {i0, i1, i2};
  for (int k = 0; k < 3; ++k) centers[k] = g_.axis[k].min + (idx[k] + 0.5) * getAxisBinWidth(k);
}

double TwoPointGrid::maxAngularScale(double scale) const {
  double a = 0;
  check(tos_grid_max_angular_scale(&g_, scale, &a));
  return a;
}

XiEstimator::XiEstimator(double scale, const TwoPointGrid& grid, BinningCoordinateType type,
                         const std::vector<Forest>& sightlines, int healpix_order, int device)
    : scale_(scale), grid_(grid) {
  build(type, sightlines, healpix_order, nullptr, device);
}

XiEstimator::XiEstimator(double scale, const TwoPointGrid& grid, BinningCoordinateType type,
                         const std::vector<Forest>& sightlines, const std::vector<tos_plate>& platelist,
                         int device)
    : scale_(scale), grid_(grid) {
  build(type, sightlines, 0, &platelist, device);
}

void XiEstimator::build(BinningCoordinateType type, const std::vector<Forest>& sightlines, int healpix_order,
                        const std::vector<tos_plate>* platelist, int device) {
  static const tos_coord_type map[3] = {TOS_POLAR, TOS_CARTESIAN, TOS_OBSERVING};
  if ((int)type < 0 || (int)type > 2 || map[type] != (tos_coord_type)grid_.desc().type)
    throw RuntimeError("coordinate type does not match the grid");
  std::vector<tos_sightline> los(sightlines.size());
  std::vector<tos_pixel> px;
  size_t total = 0;
  for (const auto& f : sightlines) total += f.pixels.size();
  px.reserve(total);
  for (size_t s = 0; s < sightlines.size(); ++s) {
    const Forest& f = sightlines[s];
    los[s].ra = f.ra;
    los[s].dec = f.dec;
    los[s].forest_id = f.forest_id;
    los[s].plate = f.plate;
    los[s].pixel_offset = px.size();
    los[s].num_pixels = (uint32_t)f.pixels.size();
    los[s].group = 0;
    for (const auto& p : f.pixels) px.push_back({p.value, p.loglam, p.weight, p.distance});
  }
  num_sightlines_ = sightlines.size();
  check(tos_engine_create(device, &engine_));
  const tos_status s =
      platelist ? tos_catalog_create_plates(engine_, los.data(), los.size(), px.data(), px.size(),
                                            platelist->data(), platelist->size(), 0.0, &catalog_)
                : tos_catalog_create(engine_, los.data(), los.size(), px.data(), px.size(), healpix_order, &catalog_);
  if (s != TOS_OK) {
    tos_engine_destroy(engine_);
    engine_ = nullptr;
    check(s);
  }
}

XiEstimator::~XiEstimator() {
  tos_catalog_destroy(catalog_);
  tos_engine_destroy(engine_);
}

void XiEstimator::run(int /*nthreads*/, bool do_cov) {
  const size_t nb = (size_t)grid_.getNBinsTotal();
  cov_.clear();
  size_t nc = 0;
  check(tos_catalog_num_cells(catalog_, &nc));
  std::vector<int64_t> ids(nc);
  check(tos_catalog_cells(catalog_, ids.data(), nc));
  xi_.assign(nb, tos_xibin{});
  std::vector<tos_xibin> cells(nc * nb);
  check(tos_xi_run(engine_, catalog_, &grid_.desc(), scale_, TOS_XI_SUBSAMPLES, xi_.data(),
                   cells.data(), &stats_));
  skybin_xis_.clear();
  for (size_t c = 0; c < nc; ++c)
    skybin_xis_[ids[c]] = std::vector<tos_xibin>(cells.begin() + c * nb, cells.begin() + (c + 1) * nb);
  tos_xibin_finalize(xi_.data(), xi_.size());
  std::cout << "Xi estimation complete!" << std::endl << std::endl;
  print_stats();
  std::cout << std::endl;
  if (do_cov) {
    // each cell's xi = didj/wgt weighted by its total wgt (XiEstimator.cc:60-97)
    std::cout << "Estimating covariance..." << std::endl;
    cov_.assign(nb * nb, 0.0);
    check(tos_xi_cell_covariance(engine_, catalog_, nullptr, cov_.data(), nullptr));
    std::cout << "Covariance estimation complete!" << std::endl << std::endl;
  }
}

void XiEstimator::save_results(const std::string& outfile) const {
  // XiEstimator::save_results (XiEstimator.cc:307-361)
  const int nb = (int)xi_.size();
  {
    std::ofstream f(outfile + ".data");
    for (int k = 0; k < nb; ++k) f << k << ' ' << lexical(xi_[k].didj) << '\n';
  }
  {
    std::ofstream f(outfile + ".details");
    std::vector<double> c(3);
    for (int k = 0; k < nb; ++k) {
      grid_.getBinCenters(k, c);
      f << k << ' ' << c[0] << ' ' << c[1] << ' ' << c[2] << ' ' << lexical(xi_[k].didj) << ' '
        << lexical(xi_[k].di) << ' ' << lexical(xi_[k].dj) << ' ' << lexical(xi_[k].wgt) << ' '
        << lexical((long long)xi_[k].num_pairs) << ' ' << lexical(xi_[k].z) << '\n';
    }
  }
  if (!cov_.empty()) {
    // upper triangle, column by column (XiEstimator.cc:334-345)
    std::ofstream f(outfile + ".cov");
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row <= col; ++row)
        f << row << ' ' << col << ' ' << lexical(cov_[(size_t)row * nb + col]) << '\n';
  }
  {
    std::ofstream f(outfile + ".iwgt");
    for (int k = 0; k < nb; ++k) f << k << ' ' << k << ' ' << lexical(1.0 / xi_[k].wgt) << '\n';
  }
}

void XiEstimator::save_subsamples(const std::string& outfile_base) const {
  // XiEstimator::save_subsamples (XiEstimator.cc:363-383)
  for (const auto& kv : skybin_xis_) {
    std::ofstream f(outfile_base + "-" + std::to_string(kv.first) + ".data");
    for (size_t k = 0; k < kv.second.size(); ++k) {
      const tos_xibin& b = kv.second[k];
      const double value = (b.wgt > 0) ? b.didj / b.wgt : 0.0;
      f << k << ' ' << lexical(value) << ' ' << lexical(b.wgt) << ' '
        << lexical((long long)b.num_pairs) << '\n';
    }
  }
}

void XiEstimator::print_stats() const {
  // XiEstimator::print_stats (XiEstimator.cc:389-408)
  const unsigned long n = num_sightlines_;
  const unsigned long total = n * (n - 1) / 2;
  std::cout << "Number of distinct los pairs " << total << std::endl;
  std::cout << "considered " << stats_.num_sightline_pairs << " of distinct los pairs. ("
            << (double)stats_.num_sightline_pairs / total << ")" << std::endl;
  std::cout << "used " << stats_.num_sightline_pairs_used << " of los pairs considered. ("
            << (double)stats_.num_sightline_pairs_used / stats_.num_sightline_pairs << ")" << std::endl;
  const unsigned long np = stats_.num_pixels;
  const unsigned long ptotal = np * (np - 1) / 2;
  std::cout << "Number of distinct pixel pairs " << ptotal << std::endl;
  std::cout << "considered " << stats_.num_pixel_pairs << " of distinct pixel pairs. ("
            << (double)stats_.num_pixel_pairs / ptotal << ")" << std::endl;
  std::cout << "used " << stats_.num_pixel_pairs_used << " of pixel pairs considered. ("
            << (double)stats_.num_pixel_pairs_used / stats_.num_pixel_pairs << ")" << std::endl;
}

}  // namespace tos
