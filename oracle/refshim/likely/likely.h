// Stand-in for deepzot likely's likely.h, with the names the reference's
// hot path uses (AbsTwoPointGrid.h:6-63, XiEstimator.cc:60-97, h5healxi.cc:138-153).
// Axes are linear "[min:max]*n" binnings: bin k covers [min + k*w, min + (k+1)*w)
// with w = (max - min)/n.  BinnedGrid's global index puts the last axis
// fastest: index = (i0 * n1 + i1) * n2 + i2, the layout the reference's hot
// loop writes directly (XiEstimator.cc:199, 249-255).
#pragma once
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "boost/smart_ptr.hpp"

namespace likely {

class RuntimeError : public std::runtime_error {
 public:
  explicit RuntimeError(std::string const& reason) : std::runtime_error(reason) {}
};

class AbsBinning {
 public:
  virtual ~AbsBinning() {}
  virtual int getNBins() const = 0;
  virtual double getBinLowEdge(int index) const = 0;
  virtual double getBinHighEdge(int index) const = 0;
  virtual double getBinWidth(int index = 0) const = 0;
  virtual double getBinCenter(int index) const { return 0.5 * (getBinLowEdge(index) + getBinHighEdge(index)); }
  virtual int getBinIndex(double value) const = 0;
};
typedef boost::shared_ptr<const AbsBinning> AbsBinningCPtr;

class UniformBinning : public AbsBinning {
 public:
  UniformBinning(double minValue, double maxValue, int nBins)
      : min_(minValue), max_(maxValue), n_(nBins), width_((maxValue - minValue) / nBins) {
    if (nBins <= 0 || !(maxValue > minValue)) throw RuntimeError("UniformBinning: bad axis");
  }
  int getNBins() const override { return n_; }
  double getBinLowEdge(int index) const override { check(index); return min_ + index * width_; }
  double getBinHighEdge(int index) const override { check(index); return min_ + (index + 1) * width_; }
  double getBinWidth(int index = 0) const override { check(index); return width_; }
  int getBinIndex(double value) const override {
    if (!(value >= min_ && value < max_)) throw RuntimeError("UniformBinning: value out of range");
    int k = static_cast<int>(std::floor((value - min_) / width_));
    return k < n_ ? k : n_ - 1;
  }

 private:
  void check(int index) const {
    if (index < 0 || index >= n_) throw RuntimeError("UniformBinning: bin index out of range");
  }
  double min_, max_;
  int n_;
  double width_;
};

class BinnedGrid {
 public:
  BinnedGrid() {}
  BinnedGrid(AbsBinningCPtr a1, AbsBinningCPtr a2, AbsBinningCPtr a3) : axes_{a1, a2, a3} {}
  int getNAxes() const { return static_cast<int>(axes_.size()); }
  AbsBinningCPtr getAxisBinning(int axis) const { return axes_.at(axis); }
  int getNBinsTotal() const {
    int n = 1;
    for (auto const& a : axes_) n *= a->getNBins();
    return n;
  }
  int getIndex(std::vector<double> const& values) const {
    int index = 0;
    for (std::size_t k = 0; k < axes_.size(); ++k) index = index * axes_[k]->getNBins() + axes_[k]->getBinIndex(values.at(k));
    return index;
  }
  void getBinCenters(int index, std::vector<double>& centers) const {
    centers.resize(axes_.size());
    for (std::size_t k = axes_.size(); k-- > 0;) {
      int n = axes_[k]->getNBins();
      centers[k] = axes_[k]->getBinCenter(index % n);
      index /= n;
    }
  }

 private:
  std::vector<AbsBinningCPtr> axes_;
};

// likely's covariance classes are not part of the reference tree; the
// accumulator here only reports that, which XiEstimator::run catches
// (XiEstimator.cc:90-93).  Runs use do_cov = false.
class CovarianceMatrix {
 public:
  bool isPositiveDefinite() const { return false; }
  double getLogDeterminant() const { return 0; }
  double getCovariance(int, int) const { return 0; }
};
typedef boost::shared_ptr<const CovarianceMatrix> CovarianceMatrixCPtr;

class CovarianceAccumulator {
 public:
  explicit CovarianceAccumulator(int) {}
  void accumulate(std::vector<double> const&, double = 1) {}
  CovarianceMatrixCPtr getCovariance() const {
    throw RuntimeError("CovarianceAccumulator: likely is not available");
  }
};

}  // namespace likely
