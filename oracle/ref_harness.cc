// ref_harness.cc — C entry point around the reference's own XiEstimator.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile (target `ref`) compiles this file together with
// the reference's unchanged sources (turbooctospice/XiEstimator.cc,
// AbsTwoPointGrid.cc, CartesianGrid.cc, PolarGrid.cc, QuasarGrid.cc,
// ThreadPool.cc) against the stand-in headers of refshim/ into
// oracle/_ref/libtosref.so.  Tests use it to pin the C oracle (xi_oracle.c)
// and the GPU engine to the reference's own arithmetic; bench.py's reference
// arm times it.  The engine never loads it.
//
// What a call does is what h5healxi does around the estimator
// (src/h5healxi.cc:163-290): build one Forest per sightline
// (types.h:56-67), bin them into HealpixBins of the given order
// (HealpixBins.h:31-43) or, in tosref_xi_plates, into PlateBins by their
// plate (PlateBins.h:18-92, its platelist read through the CCfits stand-in
// of refshim/CCfits), build the Polar/Cartesian/Quasar grid from three
// linear axes, construct XiEstimator (XiEstimator.cc:19-29) and call
// run(nthreads, false) (XiEstimator.cc:31-58).  The harness then reads the
// estimator's results: the per-cell XiBin rows skybin_xis_, their sum in
// ascending cell order with XiBin::operator+= (what xi_finalize_task does
// before it finalizes, XiEstimator.cc:298-305), the finalized xi_ and the
// five counters.  Those members are private, so this translation unit alone
// declares XiEstimator's members public while it includes XiEstimator.h; the
// class layout is unchanged.
//
// Two harness-side choices, neither of which changes the arithmetic:
//  - primary-cell subsets: a subclass of the sky bins reports only the
//    chosen cells as occupied, so run() posts a task for those cells only, while the
//    neighbour search still sees every sightline;
//  - skybin_xis_ gets one empty row per task cell before run(): each task
//    then only assigns its own existing map entry (XiEstimator.cc:156), where
//    otherwise concurrent tasks insert into one std::map with no lock, a data
//    race of the reference when nthreads > 1.
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "boost/bind.hpp"
#include "boost/function.hpp"
#include "boost/lexical_cast.hpp"
#include "boost/progress.hpp"
#include "boost/smart_ptr.hpp"
#include "boost/thread/mutex.hpp"
#include "boost/timer.hpp"
#include "healpix_map.h"
#include "likely/likely.h"

#include "RuntimeError.h"
#include "constants.h"
#include "types.h"

#define private public
#include "XiEstimator.h"
#undef private

#include "AbsTwoPointGrid.h"
#include "CartesianGrid.h"
#include "HealpixBins.h"
#include "PlateBins.h"
#include "PolarGrid.h"
#include "QuasarGrid.h"
#include "SkyBins.h"

namespace ref = turbooctospice;

namespace {

// Sky bins whose task list can be narrowed to a subset of their cells
// (HealpixBins or PlateBins): run() posts a task per occupied bin.
template <class Bins>
class Subset : public Bins {
 public:
  using Bins::Bins;
  void restrict_to(const std::vector<int>& cells) { this->occupied_bins_ = cells; }
};

// Silences std::cout (the estimator's progress and statistics) for a scope.
class QuietCout {
 public:
  QuietCout() : old_(std::cout.rdbuf(sink_.rdbuf())) {}
  ~QuietCout() { std::cout.rdbuf(old_); }

 private:
  std::ostringstream sink_;
  std::streambuf* old_;
};

void set_error(char* err, size_t cap, const std::string& msg) {
  if (err && cap) {
    std::strncpy(err, msg.c_str(), cap - 1);
    err[cap - 1] = 0;
  }
}

}  // namespace

extern "C" {

// XiBin as plain data: 7 doubles and a 64-bit count (types.h:69-121).
typedef struct {
  double didj, di, dj, wgt, wi, wj, z;
  int64_t num_pairs;
} tosref_xibin;

}  // extern "C"

namespace {

// One Forest per sightline (types.h:56-67), item = sightline index, as
// HDF5Delta::loadForests numbers them (HDF5Delta.cc:57-71).
std::vector<ref::Forest> make_sightlines(const double* ra, const double* dec, const int32_t* plate,
                                         const uint64_t* px_off, const uint32_t* npx, size_t n_los,
                                         const float* px) {
  std::vector<ref::Forest> sightlines;
  sightlines.reserve(n_los);
  for (size_t s = 0; s < n_los; ++s) {
    ref::Forest f(ra[s], dec[s], static_cast<int>(s), plate ? plate[s] : 0);
    f.pixels.reserve(npx[s]);
    for (uint32_t k = 0; k < npx[s]; ++k) {
      const float* p = px + 4 * (px_off[s] + k);
      f.pixels.push_back(ref::ForestPixel(p[0], p[1], p[2], p[3]));
    }
    sightlines.push_back(std::move(f));
  }
  return sightlines;
}

// Adds every sightline to the bins, narrows the task list, builds the grid,
// runs XiEstimator and reads its results (see tosref_xi).
template <class Bins>
long run_estimator(boost::shared_ptr<Subset<Bins> > bins, const std::vector<ref::Forest>& sightlines, int coord,
                   const double* axes, double scale, int nthreads, const int64_t* cells, size_t n_cells,
                   tosref_xibin* out_bins, tosref_xibin* out_final, tosref_xibin* out_cells,
                   int64_t* out_cell_ids, size_t cap_cells, uint64_t* counters, double* max_ang,
                   double* run_seconds) {
  for (size_t s = 0; s < sightlines.size(); ++s) bins->addItem(sightlines[s], static_cast<int>(s));
  if (cells) {
    std::vector<int> subset;
    for (size_t k = 0; k < n_cells; ++k) {
      if (!bins->checkBinExists(static_cast<int>(cells[k]))) throw std::runtime_error("subset cell not occupied");
      subset.push_back(static_cast<int>(cells[k]));
    }
    bins->restrict_to(subset);
  }
  likely::AbsBinningCPtr a[3];
  for (int k = 0; k < 3; ++k)
    a[k].reset(new likely::UniformBinning(axes[3 * k], axes[3 * k + 1], static_cast<int>(axes[3 * k + 2])));
  ref::AbsTwoPointGridPtr grid;
  ref::XiEstimator::BinningCoordinateType type;
  if (coord == 0) {
    grid.reset(new ref::PolarGrid(a[0], a[1], a[2]));
    type = ref::XiEstimator::PolarCoordinates;
  } else if (coord == 1) {
    grid.reset(new ref::CartesianGrid(a[0], a[1], a[2]));
    type = ref::XiEstimator::CartesianCoordinates;
  } else if (coord == 2) {
    grid.reset(new ref::QuasarGrid(a[0], a[1], a[2]));
    type = ref::XiEstimator::ObservingCoordinates;
  } else {
    throw std::runtime_error("bad coordinate type");
  }
  const int nb = grid->getNBinsTotal();
  ref::XiEstimator est(scale, grid, type, sightlines, bins);
  for (int c : bins->getOccupiedBins()) est.skybin_xis_[c] = std::vector<ref::XiBin>();
  const auto t0 = std::chrono::steady_clock::now();
  est.run(nthreads > 0 ? nthreads : 1, false);
  if (run_seconds) *run_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  std::vector<ref::XiBin> total(nb);
  size_t row = 0;
  for (const auto& cell : est.skybin_xis_) {
    for (int b = 0; b < nb; ++b) total[b] += cell.second[b];
    if (out_cells && row < cap_cells) {
      std::memcpy(out_cells + row * nb, cell.second.data(), sizeof(tosref_xibin) * nb);
      if (out_cell_ids) out_cell_ids[row] = cell.first;
    }
    ++row;
  }
  static_assert(sizeof(ref::XiBin) == sizeof(tosref_xibin), "XiBin layout");
  std::memcpy(out_bins, total.data(), sizeof(tosref_xibin) * nb);
  if (out_final) std::memcpy(out_final, est.xi_.data(), sizeof(tosref_xibin) * nb);
  if (counters) {
    counters[0] = est.num_sightline_pairs_;
    counters[1] = est.num_sightline_pairs_used_;
    counters[2] = est.num_pixels_;
    counters[3] = est.num_pixel_pairs_;
    counters[4] = est.num_pixel_pairs_used_;
  }
  if (max_ang) {
    max_ang[0] = est.max_ang_;
    max_ang[1] = est.cos_max_ang_;
  }
  return static_cast<long>(est.skybin_xis_.size());
}

}  // namespace

extern "C" {

// Runs the reference XiEstimator.  Inputs: sightline positions (radians),
// pixel ranges [off, off + n) of a flat pixel array of 4 floats each
// (value, loglam, weight, distance: ForestPixel order), the HEALPix order,
// the coordinate type (0 polar, 1 cartesian, 2 observing), nine axis values
// (min, max, nbins) x 3, the transverse scale and the thread count.
// cells/n_cells: NULL for every occupied cell, else the primary cells to run.
// Outputs: out_bins (n_bins raw totals), out_final (n_bins finalized, may be
// NULL), out_cells/out_cell_ids (per-cell rows in ascending cell order,
// up to cap_cells rows, may be NULL), counters[5] = num_sightline_pairs,
// num_sightline_pairs_used, num_pixels, num_pixel_pairs, num_pixel_pairs_used,
// max_ang[2] = max_ang_, cos_max_ang_, run_seconds = wall time of run() alone
// (may be NULL).  Returns the number of cells run, or -1 with a message in err.
long tosref_xi(const double* ra, const double* dec, const uint64_t* px_off, const uint32_t* npx, size_t n_los,
               const float* px, int order, int coord, const double* axes, double scale, int nthreads,
               const int64_t* cells, size_t n_cells, tosref_xibin* out_bins, tosref_xibin* out_final,
               tosref_xibin* out_cells, int64_t* out_cell_ids, size_t cap_cells, uint64_t* counters,
               double* max_ang, double* run_seconds, char* err, size_t errcap) {
  try {
    QuietCout quiet;
    const std::vector<ref::Forest> sightlines = make_sightlines(ra, dec, nullptr, px_off, npx, n_los, px);
    boost::shared_ptr<Subset<ref::HealpixBinsI> > bins(new Subset<ref::HealpixBinsI>(order));
    return run_estimator(bins, sightlines, coord, axes, scale, nthreads, cells, n_cells, out_bins, out_final,
                         out_cells, out_cell_ids, cap_cells, counters, max_ang, run_seconds);
  } catch (std::exception const& e) {
    set_error(err, errcap, e.what());
    return -1;
  }
}

// tosref_xi with the sightlines binned by BOSS plate instead of HEALPix:
// PlateBins (PlateBins.h:18-92), what h5healxi builds when its HEALPix order
// is 0 (h5healxi.cc:166-174).  plate[s] is sightline s's plate; the platelist
// (n_list rows of PLATE, RACEN, DECCEN in degrees, the columns PlateBins
// reads from the platelist FITS file) is handed to PlateBins' own
// constructor through the CCfits stand-in.  Cell ids are plate ids.
long tosref_xi_plates(const double* ra, const double* dec, const int32_t* plate, const uint64_t* px_off,
                      const uint32_t* npx, size_t n_los, const float* px, const int32_t* list_plate,
                      const float* list_racen, const float* list_deccen, size_t n_list, int coord,
                      const double* axes, double scale, int nthreads, const int64_t* cells, size_t n_cells,
                      tosref_xibin* out_bins, tosref_xibin* out_final, tosref_xibin* out_cells,
                      int64_t* out_cell_ids, size_t cap_cells, uint64_t* counters, double* max_ang,
                      double* run_seconds, char* err, size_t errcap) {
  try {
    QuietCout quiet;
    const std::vector<ref::Forest> sightlines = make_sightlines(ra, dec, plate, px_off, npx, n_los, px);
    tosref_ccfits::Table table;
    table["PLATE"].assign(list_plate, list_plate + n_list);
    table["RACEN"].assign(list_racen, list_racen + n_list);
    table["DECCEN"].assign(list_deccen, list_deccen + n_list);
    const std::string name = "tosref-platelist.fits";
    tosref_ccfits::register_table(name, table);
    boost::shared_ptr<Subset<ref::PlateBinsI> > bins(new Subset<ref::PlateBinsI>(name));
    return run_estimator(bins, sightlines, coord, axes, scale, nthreads, cells, n_cells, out_bins, out_final,
                         out_cells, out_cell_ids, cap_cells, counters, max_ang, run_seconds);
  } catch (std::exception const& e) {
    set_error(err, errcap, e.what());
    return -1;
  }
}

// HealpixBins::ang2pix (HealpixBins.h:58-66) of the stand-in map.
int64_t tosref_radec2pix(int order, double ra, double dec) {
  QuietCout quiet;
  ref::HealpixBinsI hb(order);
  return hb.ang2pix(ra, dec);
}

// Largest distance from a direction to the centre of its pixel over n
// directions (x, y, z rows), and the bound query_disc_inclusive adds.
double tosref_max_centre_distance(int order, const double* dirs, size_t n, double* bound) {
  Healpix_Map<double> m(order, RING);
  double worst = 0;
  for (size_t k = 0; k < n; ++k) {
    const double x = dirs[3 * k], y = dirs[3 * k + 1], z = dirs[3 * k + 2];
    pointing p(std::acos(z), std::atan2(y, x));
    pointing c = m.pix2ang(m.ang2pix(p));
    const double cx = std::sin(c.theta) * std::cos(c.phi), cy = std::sin(c.theta) * std::sin(c.phi),
                 cz = std::cos(c.theta);
    const double d = std::atan2(std::sqrt((y * cz - z * cy) * (y * cz - z * cy) + (z * cx - x * cz) * (z * cx - x * cz) +
                                          (x * cy - y * cx) * (x * cy - y * cx)),
                                x * cx + y * cy + z * cz);
    if (d > worst) worst = d;
  }
  if (bound) *bound = m.max_pixrad();
  return worst;
}

}  // extern "C"
