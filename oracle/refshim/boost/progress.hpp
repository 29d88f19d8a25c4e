// Stand-in for boost/progress.hpp: a progress counter that prints nothing.
#pragma once
#include <iostream>
namespace boost {
class progress_display {
 public:
  explicit progress_display(unsigned long expected, std::ostream& = std::cout) : expected_(expected) {}
  unsigned long operator++() { return ++count_; }
  unsigned long operator+=(unsigned long n) { return count_ += n; }
  unsigned long count() const { return count_; }
  unsigned long expected_count() const { return expected_; }

 private:
  unsigned long expected_ = 0, count_ = 0;
};
}  // namespace boost
