// Stand-in for boost/timer.hpp (included by XiEstimator.h, not used on the path).
#pragma once
#include <chrono>
namespace boost {
class timer {
 public:
  timer() : t0_(std::chrono::steady_clock::now()) {}
  void restart() { t0_ = std::chrono::steady_clock::now(); }
  double elapsed() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

 private:
  std::chrono::steady_clock::time_point t0_;
};
}  // namespace boost
