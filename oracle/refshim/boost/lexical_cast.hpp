// Stand-in for boost/lexical_cast.hpp: to-string conversion with the
// round-trip precision boost uses for floating point (max_digits10).
#pragma once
#include <limits>
#include <sstream>
#include <string>
#include <type_traits>
namespace boost {
template <class Target, class Source>
Target lexical_cast(const Source& s) {
  static_assert(std::is_same<Target, std::string>::value, "only conversions to std::string are used");
  std::ostringstream os;
  if (std::is_floating_point<Source>::value) os.precision(std::numeric_limits<Source>::max_digits10);
  os << s;
  return os.str();
}
}  // namespace boost
