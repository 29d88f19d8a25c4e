// xi_estimator.h — C++ host-side mirror of turbooctospice::XiEstimator
// (XiEstimator.h:17-86) on top of the C ABI: same constructor arguments,
// run / save_results / save_subsamples / print_stats, same output files.
// The pair counting itself runs on the B200 through tos_xi_run.
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tos_b200.h"

namespace tos {

// Error type of the facade (turbooctospice::RuntimeError, RuntimeError.h:8-18).
class RuntimeError : public std::runtime_error {
 public:
  explicit RuntimeError(const std::string& what) : std::runtime_error(what) {}
};

// ForestPixel (types.h:44-53) and Forest (types.h:56-67).
struct ForestPixel {
  float value, loglam, weight, distance;
};
struct Forest {
  double ra, dec;
  int forest_id, plate;
  std::vector<ForestPixel> pixels;
};

// Linear axis parsed from likely's "[min:max]*n" syntax (h5healxi.cc:43-53).
struct Axis {
  double min = 0, max = 1;
  int nbins = 1;
  static Axis parse(const std::string& spec);
};

// AbsTwoPointGrid with the coordinate type of its subclass (AbsTwoPointGrid.h:13-85).
class TwoPointGrid {
 public:
  TwoPointGrid(tos_coord_type type, const Axis& a1, const Axis& a2, const Axis& a3);
  int getNBinsTotal() const;
  int getAxisNBins(int axis) const { return g_.axis[axis].nbins; }
  double getAxisMin(int axis) const { return g_.axis[axis].min; }
  double getAxisMax(int axis) const;
  double getAxisBinWidth(int axis) const;
  void getBinCenters(int index, std::vector<double>& centers) const;
  double maxAngularScale(double scale) const;
  const tos_grid& desc() const { return g_; }

 private:
  tos_grid g_;
};

class XiEstimator {
 public:
  enum BinningCoordinateType { PolarCoordinates, CartesianCoordinates, ObservingCoordinates };
  // scale: transverse comoving scale at the minimum redshift; healpix_order:
  // the HealpixBins order (nside = 2^order); device: CUDA device id.
  XiEstimator(double scale, const TwoPointGrid& grid, BinningCoordinateType type,
              const std::vector<Forest>& sightlines, int healpix_order, int device = 0);
  // The same with the sightlines binned by plate (PlateBins, PlateBins.h:18-92):
  // platelist holds the PLATE, RACEN, DECCEN rows of the platelist file.
  XiEstimator(double scale, const TwoPointGrid& grid, BinningCoordinateType type,
              const std::vector<Forest>& sightlines, const std::vector<tos_plate>& platelist, int device = 0);
  ~XiEstimator();
  XiEstimator(const XiEstimator&) = delete;
  XiEstimator& operator=(const XiEstimator&) = delete;
  // nthreads is accepted for interface compatibility; the work runs on the GPU.
  // do_cov: also estimate the covariance of the per-cell xi (written as .cov
  // by save_results), as XiEstimator::run does (XiEstimator.cc:60-97).
  void run(int nthreads = 0, bool do_cov = false);
  void save_results(const std::string& outfile) const;
  void save_subsamples(const std::string& outfile_base) const;
  void print_stats() const;
  // finalized bins (XiBin::finalize applied) and raw per-cell sums
  const std::vector<tos_xibin>& xi() const { return xi_; }
  const std::map<int64_t, std::vector<tos_xibin>>& skybin_xis() const { return skybin_xis_; }
  const tos_xi_stats& stats() const { return stats_; }
  // covariance of the last run with do_cov (row-major n_bins x n_bins), empty otherwise
  const std::vector<double>& covariance() const { return cov_; }

 private:
  void build(BinningCoordinateType type, const std::vector<Forest>& sightlines, int healpix_order,
             const std::vector<tos_plate>* platelist, int device);
  double scale_;
  TwoPointGrid grid_;
  tos_engine* engine_ = nullptr;
  tos_catalog* catalog_ = nullptr;
  size_t num_sightlines_ = 0;
  std::vector<tos_xibin> xi_;
  std::map<int64_t, std::vector<tos_xibin>> skybin_xis_;
  tos_xi_stats stats_{};
  std::vector<double> cov_;
};

}  // namespace tos
